// Far field of the BEM matvec on sm_100a: the 12-channel screened-Coulomb
// plane-wave FMM of the reference (FMM_BEM_Octree::solve,
// src/fmm/fmm_bem_hybrid.h:183-279; operators in src/fmm/fmm.h).
//
// Channels (src/bem/node_patch.h:339-394): with a = patch area, n its normal,
// eps the dielectric ratio, charges [a f n, a h] and [a f n/eps, a h/eps]
// are screened with kappa (channels 0-7), [a f n/eps, a h] with beta0 = 1e-10
// (channels 8-11, standing in for Laplace).
//
// Every stage that is a fixed linear map runs as a dense or sparse operator
// tabulated once per problem by applying the structured kernels of the
// reference's operators (ympshift / ylcshift, ympoletoexp + yftophys,
// yphystof + yexptolocal + rotations, the L2P derivative ladders) to unit
// vectors; geometry-only bases (P2M, L2P) are tabulated the same way.  Each
// matvec then runs:
//   P2M   basis x charges, one block per childless node (yformmp)
//   M2M   per level: gather-GEMM of the children through their octant's
//         110 x 110 shift operator into per-child partials, then the partials
//         of each parent summed in child order
//   M2X   per level: gather-GEMM of the sources' multipoles through the
//         684 x 110 multipole -> 6 plane-wave operator of the parent level
//   X2L   per level: diagonal translations of each target's interaction list
//         (translate_up/down_wave, factors tabulated per offset) summed per
//         direction, then the 110 x 684 wave -> local GEMM
//   L2L   per level: gather-GEMM of the parents through the child octant's
//         shift operator, added to (or assigned) the child's locals
//   L2P   sparse derivative-expansion operator per leaf, then q(n, m) of each
//         target contracted with them (FMM_results_to_BEM,
//         src/bem/bem_kernels.cpp:12-121)
// M2X + X2L of a level run on the level's own stream as soon as its
// multipoles exist; the kernels that follow one another on a stream are
// programmatic dependent launches.  Work that cannot reach a result is not
// scheduled.  The mixed engine's two operator GEMMs (M2X, waves -> local)
// run on the 5th-generation tensor cores (tcgen05, 3xTF32, TMEM
// accumulators); the FP64 engine's on the SIMT FP64 pipe.
// Precision: T = double (FP64 engine) or float (mixed engine); tables and
// operators are computed in FP64 and rounded to T.  Expansions are stored
// [node][channel][tri(n, m)] as complex T; plane waves
// [node][direction][channel][i].
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <type_traits>
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
  const C* tcomb;        // [lg][686 combos][np_max] plane-wave translation factors
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

// ---------------------------------------------------------------- async copies
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// one 4- or 8-byte element
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem);
template <>
__device__ __forceinline__ void cp_async_elem<float>(float* smem, const float* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <>
__device__ __forceinline__ void cp_async_elem<double>(double* smem, const double* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------- P2M
// The multipole basis of a patch in its childless node (yformmp without the
// charge: i_l(beta r) P_l^m(cos theta) e^{-i m phi} * scale factors, per
// screening group) depends on geometry alone, so it is tabulated once per
// problem (p2m_basis_kernel) and every matvec only contracts it with the
// patches' 12 charges (p2m_kernel).
struct P2mItem {
  int node, level, start, count;
  int pos;  // first row of the node's patches in the basis table
  double c[3];
};

constexpr int kP2mChunk = 32;

// basis[(pos + p) * 2 + g][e] for patch p of the item, group g
// Programmatic dependent launch (PTX griddepcontrol.wait): a kernel of the
// far-field chains launched as a programmatic dependent starts as the
// previous kernel on its stream retires its CTAs and waits here until that
// grid has completed and its writes are visible.  It touches no memory
// before the wait, so every read and write keeps its order; launched
// without the attribute the instruction does nothing.  (Releasing the
// dependents at kernel start as well, griddepcontrol.launch_dependents, was
// measured slower: 0.484 against 0.447 ms a matvec -- their waiting CTAs
// hold SM slots the concurrent level streams need.)
__device__ __forceinline__ void pdl_begin() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename T>
__global__ void __launch_bounds__(64) p2m_basis_kernel(const __grid_constant__ Tables<T> tb,
                                                       const P2mItem* __restrict__ items,
                                                       const int32_t* __restrict__ contents,
                                                       const double* __restrict__ centroid,
                                                       typename C2T<T>::type* __restrict__ basis) {
  using C = typename C2T<T>::type;
  const int E = tb.E, NT = tb.nt;
  const P2mItem it = items[blockIdx.x];
  for (int t = threadIdx.x; t < 2 * it.count; t += blockDim.x) {
    const int pl = t >> 1, g = t & 1;
    const int i = contents[it.start + pl];
    const double rx = centroid[3 * i] - it.c[0], ry = centroid[3 * i + 1] - it.c[1], rz = centroid[3 * i + 2] - it.c[2];
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
    C* bs = basis + ((size_t)(it.pos + pl) * 2 + g) * E;
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
  }
}

// One block per childless node; thread (g, e) accumulates coefficient e of
// the group's channels (8 for group 0, 4 for group 1) over the node's
// patches.  Per chunk of 32 patches the basis rows (contiguous) arrive in
// shared memory by one cp.async burst while the charges are computed.
template <typename T>
__global__ void __launch_bounds__(128) p2m_kernel(const P2mItem* __restrict__ items, int E,
                                                  const int32_t* __restrict__ contents,
                                                  const double* __restrict__ area,
                                                  const double* __restrict__ normal, const double* __restrict__ eps,
                                                  const double* __restrict__ x, int n,
                                                  const typename C2T<T>::type* __restrict__ basis,
                                                  typename C2T<T>::type* __restrict__ M) {
  pdl_begin();
  using C = typename C2T<T>::type;
  __shared__ T q[kP2mChunk][kCh];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bsm = reinterpret_cast<C*>(smem_raw);  // [kP2mChunk][2][E]
  const P2mItem it = items[blockIdx.x];
  const int g = threadIdx.x >= 64 ? 1 : 0, e = threadIdx.x - 64 * g;
  const int c0 = g ? 8 : 0, nc = g ? 4 : 8;
  C acc[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c] = cmk<C>(0, 0);
  for (int base = 0; base < it.count; base += kP2mChunk) {
    const int cnt = min(kP2mChunk, it.count - base);
    __syncthreads();
    {
      const char* src = reinterpret_cast<const char*>(basis + (size_t)(it.pos + base) * 2 * E);
      const int n16 = cnt * 2 * E * (int)sizeof(C) / 16;
      for (int j = threadIdx.x; j < n16; j += blockDim.x) cp_async16(smem_raw + 16 * j, src + 16 * j);
      cp_async_commit();
    }
    if (threadIdx.x < cnt) {
      T qq[kCh];
      patch_charges<T>(area, normal, eps, x, n, contents[it.start + base + threadIdx.x], qq);
#pragma unroll
      for (int c = 0; c < kCh; ++c) q[threadIdx.x][c] = qq[c];
    }
    cp_async_wait<0>();
    __syncthreads();
    if (e < E) {
      const C* b = bsm + (size_t)g * E + e;
#pragma unroll 4
      for (int p = 0; p < cnt; ++p) {
        const C v = b[(size_t)p * 2 * E];
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < nc) {
            const T qc = q[p][c0 + c];
            acc[c].x += v.x * qc;
            acc[c].y += v.y * qc;
          }
      }
    }
  }
  if (e < E)
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (c < nc) M[((size_t)it.node * kCh + c0 + c) * E + e] = acc[c];
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

constexpr int kPairLanes = 64;  // lanes per direction pair / per target (>= nexptotp, nexptot and E)
constexpr int kM2xThreads = 3 * kPairLanes;
constexpr int kM2xChannels = 4;  // channels per M2X block (never straddles the screening groups)

// One block per (node, 4 channels); thread group g = direction pair
// (0 up/down, 1 north/south, 2 east/west) runs the pair's rotation,
// ympoletoexp and yftophys for the block's channels, the three pairs in
// parallel.  Tables are those of the node's parent level.
template <typename T>
__global__ void __launch_bounds__(kM2xThreads) m2x_kernel(const __grid_constant__ Tables<T> tb,
                                                          const M2xItem* __restrict__ items,
                                                          const typename C2T<T>::type* __restrict__ M,
                                                          typename C2T<T>::type* __restrict__ W) {
  using C = typename C2T<T>::type;
  constexpr int CB = kM2xChannels;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, NT = tb.nt, nl = tb.nl, NPM = tb.np_max;
  C* mp = reinterpret_cast<C*>(smem_raw);  // [CB][E]
  C* rot = mp + CB * E;                     // [3][CB][E]
  C* fr = rot + 3 * CB * E;                 // [3][2][CB][64]
  const M2xItem it = items[blockIdx.x / (kCh / CB)];
  const int ch0 = (blockIdx.x % (kCh / CB)) * CB;
  const int lg = 2 * (it.level - 1) + (ch0 >= 8 ? 1 : 0);
  const int nexptot = tb.nexptot[lg], np = tb.nexptotp[lg];
  const int* numphys = tb.numphys + (size_t)lg * nl;
  const T* rl = tb.rlsc + (size_t)lg * E * nl;
  const C* fexpe = tb.fexpe + tb.fexpe_off[lg];
  const C* fexpo = tb.fexpo + tb.fexpo_off[lg];
  const int g = threadIdx.x / kPairLanes, lane = threadIdx.x - g * kPairLanes;
  // after the shared multipole load the three pairs are independent: each
  // pair's 64 threads synchronise on their own named barrier
  auto pair_sync = [&]() { asm volatile("bar.sync %0, %1;\n" ::"r"(g + 1), "n"(kPairLanes) : "memory"); };
  for (int o = threadIdx.x; o < CB * E; o += blockDim.x) mp[o] = M[((size_t)it.node * kCh + ch0) * E + o];
  __syncthreads();
  // rotated multipole: pair 0 none, 1 rotate_ztoy(rdmpi2) of (-i)^m M, 2 rotate_ztox(rdpi2)
  if (lane < E) {
    const int e = lane;
    int l = 0;
    while (tri(l + 1, 0) <= e) ++l;
    const int m = e - tri(l, 0);
    for (int c = 0; c < CB; ++c) {
      const C* src = mp + c * E;
      C v;
      if (g == 0) {
        v = src[e];
      } else if (g == 1) {
        const T* rd = tb.R(ROT_MPI2);
        v = cscale(src[tri(l, 0)], tb.rd(rd, l, 0, m));
        for (int q = 1; q <= l; ++q) {
          C s = src[tri(l, q)];
          switch (q & 3) {  // (-i)^q
            case 1: s = cmk<C>(s.y, -s.x); break;
            case 2: s = cmk<C>(-s.x, -s.y); break;
            case 3: s = cmk<C>(-s.y, s.x); break;
            default: break;
          }
          v = cadd(v, cadd(cscale(s, tb.rd(rd, l, q, m)), cscale(cconj(s), tb.rd(rd, l, q, -m))));
        }
      } else {
        v = rotate_one<T>(tb, src, tb.R(ROT_PI2), l, m);
      }
      rot[(g * CB + c) * E + e] = v;
    }
  }
  pair_sync();
  // ympoletoexp: Fourier modes up (fu) and down (fd) of the pair
  if (lane < nexptot) {
    const int j = lane;
    int l = 0, ntot = 0;
    while (ntot + tb.numfour[l] <= j) {
      ntot += tb.numfour[l];
      ++l;
    }
    const int mth = j - ntot;
    const T sgn = (mth & 1) ? T(-1) : T(1);
    for (int c = 0; c < CB; ++c) {
      const C* r = rot + (g * CB + c) * E;
      C z1 = cmk<C>(0, 0), z2 = cmk<C>(0, 0);
      for (int nm = mth; nm <= NT; nm += 2) z1 = cadd(z1, cscale(r[tri(nm, mth)], rl[(size_t)tri(nm, mth) * nl + l]));
      for (int nm = mth + 1; nm <= NT; nm += 2) z2 = cadd(z2, cscale(r[tri(nm, mth)], rl[(size_t)tri(nm, mth) * nl + l]));
      fr[((g * 2 + 0) * CB + c) * 64 + j] = cadd(z1, z2);
      fr[((g * 2 + 1) * CB + c) * 64 + j] = cscale(csub(z1, z2), sgn);
    }
  }
  pair_sync();
  // yftophys of both waves of the pair
  if (lane < np) {
    const int iw = lane;
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
    for (int which = 0; which < 2; ++which)
      for (int c = 0; c < CB; ++c) {
        const C* mf = fr + ((g * 2 + which) * CB + c) * 64;
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
        const int dir = 2 * g + which;  // 0 up 1 down 2 north 3 south 4 east 5 west
        W[(((size_t)it.node * 6 + dir) * kCh + ch0 + c) * NPM + iw] = val;
      }
  }
}

// ---------------------------------------------------------------- X2L
// X2L is split in two.  xl_translate_kernel applies the diagonal plane-wave
// translations (translate_up/down_wave) of every target's interaction list
// and leaves, per (target, channel), the six accumulated waves as 6 x 2NPM
// reals in the ACC scratch.  The conversion of those waves to a local
// expansion (yphystof, yexptolocal, rotate_ytoz / rotate_ztox back, sum of
// the three direction pairs) is R-linear and fixed per (level, screening
// group): it is tabulated once per problem by xl_convert_basis_kernel and
// applied by op_gemm_kernel.
struct XlTarget {
  int node, acc_row;             // target node; its row block of the ACC scratch
  int first_entry, n_entries;    // interactions sorted by direction
  int dir_start[7];              // direction d: entries [first + dir_start[d], first + dir_start[d + 1])
};
// One diagonal translation: source node, direction, and the translation
// factor's index combo = up * 343 + (a+3) * 49 + (b+3) * 7 + (c+3) with
// (a, b, c) the source->target offset in the direction's rotated frame.
struct XlEntry {
  int src;
  short combo;
  signed char dir, pad;
};
constexpr int kCombos = 686;
constexpr int kXlChannels = 4;                    // channels per translate block (one screening group)
constexpr int kXlUnroll = 2;

constexpr int kXlGroups = 7;                     // lane groups of a translate block
constexpr int kXlDirThreads = kXlGroups * kPairLanes;

// One block per (target, 4 channels); thread (lane group g, lane i = plane
// wave) sums W[src][d][ch][i] * factor[combo][i] over its share of the
// target's entries, in registers.  The entries are sorted by direction and
// the seven lane groups take equal contiguous slices of them, whatever the
// mix of directions (it depends on the target's surroundings).  A slice
// leaves one partial sum per direction it meets, in shared slot g + d (the
// pairs (g, d) met along the list have distinct g + d, at most 12 of them);
// then each direction's partials are added in group order (deterministic)
// and ACC[acc_row][ch][d][i] (re, im) is stored for all six directions, 0
// for one without entries.
constexpr int kXlSlots = kXlGroups + 5;
template <typename T>
__global__ void __launch_bounds__(kXlDirThreads, 2) xl_translate_kernel(const __grid_constant__ Tables<T> tb,
                                                                        int parent_level,
                                                                        const XlTarget* __restrict__ targets,
                                                                        int n_targets,
                                                                        const XlEntry* __restrict__ entries,
                                                                        const typename C2T<T>::type* __restrict__ W,
                                                                        typename C2T<T>::type* __restrict__ ACC) {
  pdl_begin();
  using C = typename C2T<T>::type;
  constexpr int CB = kXlChannels;
  constexpr int U = kXlUnroll;  // entries in flight per thread (measured: 2 beats 4, 6 and 8 spill)
  __shared__ C part[kXlSlots][CB][kPairLanes];
  const int NPM = tb.np_max;
  const int t = blockIdx.x / (kCh / CB);
  const int ch0 = (blockIdx.x % (kCh / CB)) * CB;
  const int g = threadIdx.x / kPairLanes, i = threadIdx.x - g * kPairLanes;
  const int lg = 2 * parent_level + (ch0 >= 8 ? 1 : 0);
  const XlTarget tg = targets[t];  // t < n_targets: the grid has one block set per target
  const int np = tb.nexptotp[lg];
  const bool live = i < NPM && i < np;  // plane waves beyond this level's count stay 0
  const C* tc = tb.tcomb + (size_t)lg * kCombos * NPM + i;
  // sum over entries [b, e) of direction d
  auto accum = [&](int d, int b, int e, C (&a)[CB]) {
#pragma unroll
    for (int c = 0; c < CB; ++c) a[c] = cmk<C>(0, 0);
    if (!live) return;
    const XlEntry* ent = entries + tg.first_entry;
    const C* Wd = W + ((size_t)d * kCh + ch0) * NPM + i;
    for (int k0 = b; k0 < e; k0 += U) {
      int src[U], combo[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const XlEntry en = ent[min(k0 + u, e - 1)];
        src[u] = en.src;
        combo[u] = en.combo;
      }
      C tt[U], w[U][CB];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        tt[u] = tc[(size_t)combo[u] * NPM];
#pragma unroll
        for (int c = 0; c < CB; ++c) w[u][c] = Wd[((size_t)src[u] * 6 * kCh + c) * NPM];
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (k0 + u < e)
#pragma unroll
          for (int c = 0; c < CB; ++c) a[c] = cadd(a[c], cmul(w[u][c], tt[u]));
    }
  };
  // slice [gb, ge) of the target's entries
  const int n = tg.n_entries;
  const int gb = (int)(((long long)g * n) / kXlGroups), ge = (int)(((long long)(g + 1) * n) / kXlGroups);
  for (int d = 0; d < 6; ++d) {
    const int b = max(gb, tg.dir_start[d]), e = min(ge, tg.dir_start[d + 1]);
    if (b >= e) continue;
    C a[CB];
    accum(d, b, e, a);
#pragma unroll
    for (int c = 0; c < CB; ++c) part[g + d][c][i] = a[c];
  }
  __syncthreads();
  if (g < 6 && i < NPM) {
    // direction g: the slices that meet its entries, in order
    const int d = g, b = tg.dir_start[d], e = tg.dir_start[d + 1];
    C a[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) a[c] = cmk<C>(0, 0);
    if (b < e) {
      const int g0 = (int)(((long long)b * kXlGroups) / max(n, 1));
      for (int gg = max(g0 - 1, 0); gg < kXlGroups; ++gg) {
        const int sb = (int)(((long long)gg * n) / kXlGroups), se = (int)(((long long)(gg + 1) * n) / kXlGroups);
        if (se <= b) continue;
        if (sb >= e) break;
        if (max(sb, b) >= min(se, e)) continue;
#pragma unroll
        for (int c = 0; c < CB; ++c) a[c] = cadd(a[c], part[gg + d][c][i]);
      }
    }
    C* out = ACC + (((size_t)tg.acc_row * kCh + ch0) * 6 + d) * NPM + i;
#pragma unroll
    for (int c = 0; c < CB; ++c) out[(size_t)c * 6 * NPM] = a[c];
  }
  (void)n_targets;
}

// Conversion of one accumulated-wave vector to a local expansion, applied
// to unit vectors: block (b, g) computes column b of the conversion operator
// of screening group g for targets below parent_level, written as
// ops[lg][b][r] (r < 2E real components, rows padded to RP).
template <typename T>
__global__ void __launch_bounds__(kPairLanes) xl_convert_basis_kernel(const __grid_constant__ Tables<T> tb,
                                                                      int parent_level, int RP,
                                                                      T* __restrict__ ops) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, nl = tb.nl, NPM = tb.np_max, K = 12 * NPM;
  C* acc = reinterpret_cast<C*>(smem_raw);  // [6 dirs][NPM]
  C* loc = acc;                              // [3 pairs][E], reuses acc after yphystof
  C* mf = acc + 6 * NPM;                     // [6][64]
  const int b = blockIdx.x % K, g = blockIdx.x / K;
  const int lg = 2 * parent_level + g;
  const int lane = threadIdx.x;
  const int nexptot = tb.nexptot[lg];
  for (int o = lane; o < 6 * NPM; o += blockDim.x) acc[o] = cmk<C>(0, 0);
  __syncthreads();
  if (lane == 0) {
    const int dir = b / (2 * NPM), rem = b % (2 * NPM);
    acc[dir * NPM + rem / 2] = (rem & 1) ? cmk<C>(0, 1) : cmk<C>(1, 0);
  }
  __syncthreads();
  const int* numphys = tb.numphys + (size_t)lg * nl;
  const C* fb = tb.fexpback + tb.fexpback_off[lg];
  const T* rl = tb.rlsc + (size_t)lg * E * nl;
  // yphystof of the six waves
  if (lane < nexptot) {
    const int j = lane;
    int l = 0, nftot = 0, nptot = 0, bb = 0;
    while (nftot + tb.numfour[l] <= j) {
      nftot += tb.numfour[l];
      nptot += numphys[l] / 2;
      bb += (tb.numfour[l] - 1) * (numphys[l] / 2);
      ++l;
    }
    const int mm = j - nftot + 1;
    const int na = numphys[l], na2 = na / 2;
    const T ina = T(1) / T(na);
    const int nodd = (tb.numfour[l] - 1) / 2;
    for (int d = 0; d < 6; ++d) {
      const C* ph = acc + (size_t)d * NPM + nptot;
      C sum = cmk<C>(0, 0);
      if (mm == 1) {
        for (int iv = 0; iv < na2; ++iv) sum.x += T(2) * ph[iv].x;
      } else if (mm & 1) {
        const C* f = fb + bb + ((mm - 3) / 2) * na2;
        for (int iv = 0; iv < na2; ++iv) sum = cadd(sum, cscale(f[iv], T(2) * ph[iv].x));
      } else {
        const C* f = fb + bb + nodd * na2 + ((mm - 2) / 2) * na2;
        for (int iv = 0; iv < na2; ++iv) sum = cadd(sum, cmul(f[iv], cmk<C>(0, T(2) * ph[iv].y)));
      }
      mf[(size_t)d * 64 + j] = cscale(sum, ina);
    }
  }
  __syncthreads();
  // yexptolocal per pair
  if (lane < E) {
    const int e = lane;
    int nm = 0;
    while (tri(nm + 1, 0) <= e) ++nm;
    const int mth = e - tri(nm, 0);
    const T rs = T(3.14159265358979323846) / (tb.betascal[lg] * T(2)) * tb.sfac[e];
    for (int pg = 0; pg < 3; ++pg) {
      const C* fu = mf + (size_t)(2 * pg) * 64;
      const C* fd = mf + (size_t)(2 * pg + 1) * 64;
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
      v = cscale(v, rs);
      switch (mth & 3) {  // * i^m
        case 1: v = cmk<C>(-v.y, v.x); break;
        case 2: v = cmk<C>(-v.x, -v.y); break;
        case 3: v = cmk<C>(v.y, -v.x); break;
        default: break;
      }
      loc[(size_t)pg * E + e] = v;
    }
  }
  __syncthreads();
  // rotate back and sum the pairs
  if (lane < E) {
    const int e = lane;
    int l = 0;
    while (tri(l + 1, 0) <= e) ++l;
    const int m = e - tri(l, 0);
    const C v0 = loc[e];
    C v1 = rotate_one<T>(tb, loc + E, tb.R(ROT_PI2), l, m);
    switch (m & 3) {  // rotate_ytoz: * i^m
      case 1: v1 = cmk<C>(-v1.y, v1.x); break;
      case 2: v1 = cmk<C>(-v1.x, -v1.y); break;
      case 3: v1 = cmk<C>(v1.y, -v1.x); break;
      default: break;
    }
    const C v2 = rotate_one<T>(tb, loc + 2 * E, tb.R(ROT_MPI2), l, m);
    const C v = cadd(cadd(v0, v1), v2);
    T* col = ops + ((size_t)lg * K + b) * RP;
    col[2 * e] = v.x;
    col[2 * e + 1] = v.y;
  }
  for (int r = 2 * E + lane; r < RP; r += blockDim.x) ops[((size_t)lg * K + b) * RP + r] = 0;
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

constexpr int kEvalChunk = 32;  // targets per l2p_eval block

// q(n, m) = i_n(beta r) P_n^m(cos theta) e^{i m phi} of every target patch
// relative to its leaf centre, n <= nt + 2, per screening group: geometry
// alone, tabulated once per problem as Q[item][g][tri(n, m)][lane].
template <typename T>
__global__ void __launch_bounds__(kEvalChunk) l2p_basis_kernel(const __grid_constant__ Tables<T> tb,
                                                               const LeafItem* __restrict__ items,
                                                               const int32_t* __restrict__ contents,
                                                               const double* __restrict__ centroid,
                                                               typename C2T<T>::type* __restrict__ Q) {
  using C = typename C2T<T>::type;
  const int NT = tb.nt, N2 = NT + 2;
  const int EQ = (NT + 3) * (NT + 4) / 2;
  const LeafItem it = items[blockIdx.x];
  const int k = threadIdx.x;
  if (k >= it.count) return;
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
  T bi[kMaxNT + 4];
  for (int g = 0; g < 2; ++g) {
    const int lg = 2 * it.level + g;
    bessel_in_dev<T>(tb.scale[lg], (T)(d * (double)tb.beta[g]), N2, bi);
    C* q = Q + ((size_t)blockIdx.x * 2 + g) * EQ * kEvalChunk + k;
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
        q[(size_t)tri(nn, m) * kEvalChunk] = cscale(em, amp);
      }
    }
  }
}

// One block per chunk of <= 64 targets of a leaf; thread (slice s, target k)
// sums a quarter of the terms (s = 2 g + half: screening group g, half of
// the tri(n, m) range) of f = Re sum q F, h_j = Re sum q H_j (F only to
// n <= nt+1); the four partial sums are added in a fixed order and
// y_f = f / 4 pi, y_h = n . h / 4 pi assigned to the far-field buffer.
constexpr int kEvalThreads = 4 * kEvalChunk;

template <typename T>
__global__ void __launch_bounds__(kEvalThreads) l2p_eval_kernel(int nt, const LeafItem* __restrict__ items,
                                                                const int32_t* __restrict__ contents,
                                                                const double* __restrict__ normal,
                                                                const typename C2T<T>::type* __restrict__ D,
                                                                const typename C2T<T>::type* __restrict__ Q, int n,
                                                                double* __restrict__ y) {
  pdl_begin();
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int EQ = (nt + 3) * (nt + 4) / 2, EF = (nt + 2) * (nt + 3) / 2;
  C* Ds = reinterpret_cast<C*>(smem_raw);                   // [2][4][EQ]
  T* part = reinterpret_cast<T*>(Ds + 8 * EQ);              // [4 slices][4 sums][kEvalChunk]
  // FP32: the item's whole basis block (contiguous, 80 KB) is copied into
  // shared memory in one cp.async burst, so every load is in flight at once
  constexpr bool kStageQ = sizeof(T) == 4;
  C* Qs = reinterpret_cast<C*>(part + 16 * kEvalChunk);     // [2][EQ][kEvalChunk]
  const LeafItem it = items[blockIdx.x];
  const C* Qb = Q + (size_t)blockIdx.x * 2 * EQ * kEvalChunk;
  if (kStageQ) {
    const char* src = reinterpret_cast<const char*>(Qb);
    char* dst = reinterpret_cast<char*>(Qs);
    const int n16 = 2 * EQ * kEvalChunk * (int)sizeof(C) / 16;
    for (int j = threadIdx.x; j < n16; j += blockDim.x) cp_async16(dst + 16 * j, src + 16 * j);
    cp_async_commit();
  }
  for (int o = threadIdx.x; o < 8 * EQ; o += blockDim.x) Ds[o] = D[(size_t)it.leaf * 8 * EQ + o];
  if (kStageQ) cp_async_wait<0>();
  __syncthreads();
  const int s = threadIdx.x / kEvalChunk, k = threadIdx.x - s * kEvalChunk;
  const int g = s >> 1, half = EQ / 2;
  const int e0 = (s & 1) ? half : 0, e1 = (s & 1) ? EQ : half;
  T f = 0, h0 = 0, h1 = 0, h2 = 0;
  if (k < it.count) {
    const C* q = (kStageQ ? Qs : Qb) + (size_t)g * EQ * kEvalChunk + k;
    const C* F = Ds + g * 4 * EQ;
#pragma unroll 8
    for (int e = e0; e < e1; ++e) {
      const C v = q[(size_t)e * kEvalChunk];
      if (e < EF) f += v.x * F[e].x - v.y * F[e].y;
      h0 += v.x * F[EQ + e].x - v.y * F[EQ + e].y;
      h1 += v.x * F[2 * EQ + e].x - v.y * F[2 * EQ + e].y;
      h2 += v.x * F[3 * EQ + e].x - v.y * F[3 * EQ + e].y;
    }
  }
  part[(s * 4 + 0) * kEvalChunk + k] = f;
  part[(s * 4 + 1) * kEvalChunk + k] = h0;
  part[(s * 4 + 2) * kEvalChunk + k] = h1;
  part[(s * 4 + 3) * kEvalChunk + k] = h2;
  __syncthreads();
  if (s != 0 || k >= it.count) return;
  T sum[4];
  for (int j = 0; j < 4; ++j)
    sum[j] = ((part[(0 * 4 + j) * kEvalChunk + k] + part[(1 * 4 + j) * kEvalChunk + k]) +
              part[(2 * 4 + j) * kEvalChunk + k]) + part[(3 * 4 + j) * kEvalChunk + k];
  const int i = contents[it.start + k];
  const double k4 = 0.07957747154594767;
  const double h = normal[3 * i] * (double)sum[1] + normal[3 * i + 1] * (double)sum[2] +
                   normal[3 * i + 2] * (double)sum[3];
  y[i] = (double)sum[0] * k4;  // far-field buffer: every patch is in exactly one leaf
  y[n + i] = h * k4;
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
  const int RP = (R + 3) & ~3;
  T* col = ops + ((size_t)op * R + k) * RP;  // column k: [op][k][r], rows padded to RP with zeros
  for (int o = threadIdx.x; o < E; o += blockDim.x) {
    col[2 * o] = acc[o].x;
    col[2 * o + 1] = acc[o].y;
  }
  for (int r = R + threadIdx.x; r < RP; r += blockDim.x) col[r] = 0;
}

// Operator form of M2M and L2L as a gather-GEMM.  A tile is up to 16
// columns sharing one operator (kind, level, screening group, octant); a
// column is (source node, destination row, channel).  M2M writes one
// partial per (parent, child) and shift_reduce_kernel sums a parent's
// partials in child order; L2L writes the child's local expansion directly
// (assigned, or added to the X2L result).
struct ShiftTile {
  int op;  // operator index including the screening-group offset
  int first_col, n_cols;
};
struct ShiftCol {
  int src, dst, ch, accumulate;
};
struct ShiftReduce {
  int parent, first_slot, n_slots;
};
constexpr int kTileCols = 64;   // columns per shift tile: the operator load is shared by all of them
constexpr int kGemmThreads = (112 / 4) * (kTileCols / 4);  // 4 x 4 outputs per thread, R <= 112

template <typename T>
__device__ __forceinline__ void load4(const T* p, T (&v)[4]);
template <>
__device__ __forceinline__ void load4<float>(const float* p, float (&v)[4]) {
  const float4 u = *reinterpret_cast<const float4*>(p);
  v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
}
template <>
__device__ __forceinline__ void load4<double>(const double* p, double (&v)[4]) {
  const double2 u = reinterpret_cast<const double2*>(p)[0], w = reinterpret_cast<const double2*>(p)[1];
  v[0] = u.x, v[1] = u.y, v[2] = w.x, v[3] = w.y;
}

// One block per tile; thread (row group rg, column group cg) computes rows
// 4rg..4rg+3 of columns 4cg..4cg+3: Y[dst][ch] (= or +=) A_op X[src][ch].
// The operator (its transpose, rows padded to RP) arrives in shared memory
// in one cp.async burst while the tile's inputs are gathered.
template <typename T>
__global__ void __launch_bounds__(kGemmThreads) shift_gemm_kernel(int E, const ShiftTile* __restrict__ tiles,
                                                                  const ShiftCol* __restrict__ cols,
                                                                  const T* __restrict__ ops,
                                                                  const T* __restrict__ X, T* __restrict__ Y) {
  pdl_begin();
  const int R = 2 * E, RP = (R + 3) & ~3;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);  // [R][RP]
  T* xs = As + (size_t)R * RP;              // [R][kTileCols]
  const ShiftTile tl = tiles[blockIdx.x];
  {
    const char* src = reinterpret_cast<const char*>(ops + (size_t)tl.op * R * RP);
    char* dst = reinterpret_cast<char*>(As);
    const int n16 = R * RP * (int)sizeof(T) / 16;
    for (int j = threadIdx.x; j < n16; j += blockDim.x) cp_async16(dst + 16 * j, src + 16 * j);
    cp_async_commit();
  }
  // columns: asynchronous element copies, column-fastest so that the
  // shared-memory writes of a warp fall in distinct banks
  for (int o = threadIdx.x; o < kTileCols * R; o += blockDim.x) {
    const int j = o % kTileCols, k = o / kTileCols;
    if (j < tl.n_cols) {
      const ShiftCol c = cols[tl.first_col + j];
      cp_async_elem(xs + k * kTileCols + j, X + ((size_t)c.src * kCh + c.ch) * R + k);
    } else {
      xs[k * kTileCols + j] = 0;
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int ngr = RP / 4;
  if (threadIdx.x >= ngr * (kTileCols / 4)) return;
  const int rg = threadIdx.x % ngr, cg = threadIdx.x / ngr;
  if (4 * cg >= tl.n_cols) return;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0;
  const T* a = As + 4 * rg;
  const T* x = xs + 4 * cg;
#pragma unroll 10
  for (int k = 0; k < R; ++k) {
    T av[4], xv[4];
    load4<T>(a + (size_t)k * RP, av);
    load4<T>(x + k * kTileCols, xv);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] += av[i] * xv[j];
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (4 * cg + j >= tl.n_cols) break;
    const ShiftCol c = cols[tl.first_col + 4 * cg + j];
    T* y = Y + ((size_t)c.dst * kCh + c.ch) * R;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = 4 * rg + i;
      if (r < R) y[r] = c.accumulate ? y[r] + acc[i][j] : acc[i][j];
    }
  }
}

// Dense operator applied to gathered columns: Y[col] = A_op X[col] for the
// multipole -> plane-wave map (684 x 110 per level and screening group) and
// the accumulated-wave -> local map (110 x 684).  A tile is 112 rows of one
// operator by up to 32 columns; K streams through shared memory in chunks
// (cp.async, double-buffered); thread (rg, cg) owns rows 4rg..4rg+3 and
// columns 8cg..8cg+7.  Output row r of column c goes to
// Y[dst_c + (r / seg) * seg_stride + r % seg].
struct GemmTile {
  int op, first_col, n_cols, row0;
  int kc0, nkc;        // tensor-core tiles: k chunks [kc0, kc0 + nkc) of the operator
  long long dst_off;   // added to every column's output offset (split-K partial slot)
};
struct GemmCol {
  long long src, dst;  // element offsets of the column's input vector and output base
};
constexpr int kOpRows = 112;
constexpr int kOpCols = 32;
constexpr int kOpThreads = (kOpRows / 4) * (kOpCols / 8);

template <typename T>
struct OpChunk;  // K rows per pipeline stage
template <>
struct OpChunk<float> {
  static constexpr int value = 56;
};
template <>
struct OpChunk<double> {
  static constexpr int value = 28;
};


template <typename T>
__global__ void __launch_bounds__(kOpThreads) op_gemm_kernel(const GemmTile* __restrict__ tiles,
                                                             const GemmCol* __restrict__ cols,
                                                             const T* __restrict__ ops, int K, int RP, int R,
                                                             int seg, long long seg_stride,
                                                             const T* __restrict__ X, T* __restrict__ Y) {
  pdl_begin();
  constexpr int KC = OpChunk<T>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);  // [2][KC][kOpRows]
  T* xs = As + 2 * KC * kOpRows;            // [2][KC][kOpCols]
  const GemmTile tl = tiles[blockIdx.x];
  const T* A0 = ops + (size_t)tl.op * K * RP + tl.row0;
  const int nchunks = (K + KC - 1) / KC;
  auto stage = [&](int c, int buf) {
    const int kb = c * KC, kn = min(KC, K - kb);
    T* a = As + (size_t)buf * KC * kOpRows;
    constexpr int per16 = 16 / (int)sizeof(T), chunks = kOpRows / per16;  // 16-byte copies per row
    for (int j = threadIdx.x; j < kn * chunks; j += blockDim.x) {
      const int k = j / chunks, q = j - k * chunks;
      cp_async16(a + k * kOpRows + per16 * q, A0 + (size_t)(kb + k) * RP + per16 * q);
    }
    T* x = xs + (size_t)buf * KC * kOpCols;
    for (int j = threadIdx.x; j < kn * kOpCols; j += blockDim.x) {
      const int k = j / kOpCols, n = j - k * kOpCols;
      if (n < tl.n_cols)
        cp_async_elem<T>(x + k * kOpCols + n, X + cols[tl.first_col + n].src + kb + k);
      else
        x[k * kOpCols + n] = 0;
    }
    cp_async_commit();
  };
  const int rg = threadIdx.x % (kOpRows / 4), cg = threadIdx.x / (kOpRows / 4);
  T acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0;
  stage(0, 0);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      stage(c + 1, (c + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int kn = min(KC, K - c * KC);
    const T* a = As + (size_t)(c & 1) * KC * kOpRows + 4 * rg;
    const T* x = xs + (size_t)(c & 1) * KC * kOpCols + 8 * cg;
#pragma unroll 4
    for (int k = 0; k < kn; ++k) {
      T av[4], x0[4], x1[4];
      load4<T>(a + k * kOpRows, av);
      load4<T>(x + k * kOpCols, x0);
      load4<T>(x + k * kOpCols + 4, x1);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j] += av[i] * x0[j];
          acc[i][4 + j] += av[i] * x1[j];
        }
      }
    }
    __syncthreads();  // buffer (c & 1) is refilled by the stage of chunk c + 2
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int n = 8 * cg + j;
    if (n >= tl.n_cols) break;
    const long long dst = cols[tl.first_col + n].dst;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = tl.row0 + 4 * rg + i;
      if (r < R) Y[dst + (long long)(r / seg) * seg_stride + r % seg] = acc[i][j];
    }
  }
}

// ---------------------------------------------------------------- tensor-core operator GEMM
// The same gathered GEMM on the 5th-generation tensor cores for the FP32
// engine: tcgen05.mma kind::tf32 with FP32 accuracy from the 3xTF32 split
// (A = A_hi + A_lo, X = X_hi + X_lo, A X ~ A_hi X_hi + A_hi X_lo + A_lo X_hi,
// hi = the value with its 13 low mantissa bits cleared).  A CTA owns 128
// operator rows x 128 columns; K streams in chunks of 32 through two
// shared-memory stages; the accumulator lives in tensor memory (128 lanes x
// 128 columns FP32).  Operands are K-major in the no-swizzle canonical
// layout: 16-byte core rows (4 values of k), row r of an 8-row group at
// 16 r bytes, 8-row groups 128 bytes apart, the two 16-byte k halves of one
// MMA step a full 128-row panel apart.  The operator's hi and lo halves are
// stored in global memory already in that layout, one 32 KB block per
// (operator, row tile, k chunk).
namespace tc {

constexpr int kRows = 128, kKC = 32, kThreads = 128;
// tile widths: multipole -> waves (K = 110, many columns) and waves -> local
// (K = 684, fewer columns: narrower tiles give more CTAs)
constexpr int kColsM2x = 64, kColsXl = 64;
constexpr int kPanel = kRows * 16;                  // bytes of one 4-wide k panel of 128 rows
constexpr int kHalf = kKC / 4 * kPanel;             // bytes of the operator's hi (or lo) part of a chunk: 16 KB
// dynamic shared memory of a tile NC columns wide: two stages of operator
// and column chunks, and the column tables
constexpr int smem_bytes(int nc) { return 2 * (2 * kHalf + 2 * (kKC / 4 * nc * 16)) + 16 * nc; }
constexpr long long kWaitCycles = 2000000000LL;     // about one second at the boost clock
constexpr long long kStallCycles = 200000LL;        // bound of the timeout test's wait (about 0.1 ms)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// shared-memory matrix descriptor: start, leading (k-half) and stride
// (8-row group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// bounded wait for a barrier phase; false after `limit` cycles (by default
// about a second)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit = kWaitCycles) {
  const long long t0 = clock64();
  while (!mbar_try(bar, phase))
    if (clock64() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ float hi_part(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace tc

// Y[dst_n + (r / seg) * seg_stride + r % seg] = sum_k A_op[r][k] X[src_n + k]
// for the 128 rows of the tile's row block and its <= NC columns.  packed
// holds [op][row tile][k chunk] blocks of [hi, lo][8 panels][128 rows][4].
// Software pipeline over two shared-memory stages: right after thread 0
// issues the MMAs of chunk c, all threads start the operator copy
// (cp.async) and the column loads (into registers) of chunk c + 1, so the
// loads overlap the tensor-core work; the columns are split into hi / lo
// when they are stored.  Every wait is bounded and a timeout sets status[0]
// (the kernel stops issuing, still waits, with the full bound, for the MMAs
// it committed, skips its store and frees its tensor memory).  status[1] != 0
// is the timeout test: the first pipeline step of every CTA also waits, with
// a short bound, on a barrier that nothing arrives on, so that wait always
// runs out and the timeout path runs.
template <int NC>
__global__ void __launch_bounds__(tc::kThreads, 1) op_gemm_tc_kernel(
    const GemmTile* __restrict__ tiles, const GemmCol* __restrict__ cols, const float* __restrict__ packed,
    int n_mtiles, int n_chunks, int K, int R, int seg, long long seg_stride, const float* __restrict__ X,
    float* __restrict__ Y, int* __restrict__ status) {
  pdl_begin();
  static_assert(NC % 32 == 0 && NC >= 32 && NC <= 256, "tile width");
  constexpr int kXHalf = tc::kKC / 4 * NC * 16;     // bytes of the columns' hi (or lo) part of a chunk
  constexpr int kStageB = 2 * tc::kHalf + 2 * kXHalf;
  constexpr int kGroups = NC / 32;                  // 8-column groups per warp
  extern __shared__ __align__(1024) unsigned char smem_tc[];
  __shared__ __align__(8) uint64_t bars[3];  // [0], [1]: MMA completion per stage; [2]: never arrived on
  __shared__ uint32_t tmem_slot;
  const bool stall_test = status[1] != 0;
  long long* dsts = reinterpret_cast<long long*>(smem_tc + 2 * kStageB);  // [NC]
  long long* srcs = dsts + NC;                                            // [NC]
  const GemmTile tl = tiles[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int n = tid; n < NC; n += tc::kThreads) {
    long long sv = -1, dv = 0;
    if (n < tl.n_cols) {
      const GemmCol cl = cols[tl.first_col + n];
      sv = cl.src;
      dv = cl.dst;
    }
    srcs[n] = sv;
    dsts[n] = dv;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_slot)),
                 "r"(NC));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    tc::mbar_init(&bars[0]);
    tc::mbar_init(&bars[1]);
    tc::mbar_init(&bars[2]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NC >> 3) << 17) |
                         ((uint32_t)(tc::kRows >> 4) << 24);
  const int mt = tl.row0 / tc::kRows;
  const char* ablk = reinterpret_cast<const char*>(packed) + (size_t)(tl.op * n_mtiles + mt) * n_chunks * 2 * tc::kHalf;
  // lane (j, u) of warp w handles column n = 8 (w + 4 gi) + j and k = 4q + u
  const int u = lane & 3;
  float xr[kGroups][tc::kKC / 4];
  auto issue = [&](int i) {  // local chunk i = operator chunk kc0 + i
    const int c = tl.kc0 + i;
    unsigned char* st = smem_tc + (i & 1) * kStageB;
    const char* ga = ablk + (size_t)c * 2 * tc::kHalf;
    for (int j = tid; j < 2 * tc::kHalf / 16; j += tc::kThreads) cp_async16(st + 16 * j, ga + 16 * j);
    cp_async_commit();
    const int kb = c * tc::kKC;
#pragma unroll
    for (int gi = 0; gi < kGroups; ++gi) {
      const long long sv = srcs[8 * (warp + 4 * gi) + (lane >> 2)];
#pragma unroll
      for (int q = 0; q < tc::kKC / 4; ++q) {
        const int k = kb + 4 * q + u;
        xr[gi][q] = (sv >= 0 && k < K) ? X[sv + k] : 0.f;
      }
    }
  };
  __syncthreads();  // column tables visible before the first gather
  issue(0);
  bool ok = true;
  int last = -1;  // last local chunk whose MMAs were committed
  for (int c = 0; c < tl.nkc; ++c) {
    unsigned char* st = smem_tc + (c & 1) * kStageB;
    float* xh = reinterpret_cast<float*>(st + 2 * tc::kHalf);
    float* xl = reinterpret_cast<float*>(st + 2 * tc::kHalf + kXHalf);
    // after a timed-out wait the stage may still be read by MMAs in flight:
    // nothing is written to it
    if (ok) {
#pragma unroll
      for (int gi = 0; gi < kGroups; ++gi) {
        const int n = 8 * (warp + 4 * gi) + (lane >> 2);
#pragma unroll
        for (int q = 0; q < tc::kKC / 4; ++q) {
          const float h = tc::hi_part(xr[gi][q]);
          xh[(q * NC + n) * 4 + u] = h;
          xl[(q * NC + n) * 4 + u] = xr[gi][q] - h;
        }
      }
    }
    cp_async_wait<0>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = tc::smem_u32(st), x0 = a0 + 2 * tc::kHalf;
#pragma unroll
      for (int ks = 0; ks < tc::kKC / 8; ++ks) {
        const uint32_t offa = (uint32_t)ks * 2 * tc::kPanel, offx = (uint32_t)ks * 2 * NC * 16;
        const uint64_t ah = tc::desc(a0 + offa, tc::kPanel, 128);
        const uint64_t al = tc::desc(a0 + tc::kHalf + offa, tc::kPanel, 128);
        const uint64_t bh = tc::desc(x0 + offx, NC * 16, 128);
        const uint64_t bl = tc::desc(x0 + kXHalf + offx, NC * 16, 128);
        tc::mma_tf32(tmem, ah, bh, idesc, (c > 0 || ks > 0) ? 1u : 0u);
        tc::mma_tf32(tmem, ah, bl, idesc, 1u);
        tc::mma_tf32(tmem, al, bh, idesc, 1u);
      }
      tc::commit(&bars[c & 1]);
    }
    last = c;
    if (c + 1 < tl.nkc) {
      // stage (c + 1) & 1 was read by the MMAs of chunk c - 1
      if (c >= 1 && !tc::mbar_wait(&bars[(c + 1) & 1], (uint32_t)(((c - 1) >> 1) & 1))) ok = false;
      if (c == 1 && stall_test && !tc::mbar_wait(&bars[2], 0u, tc::kStallCycles)) ok = false;
      if (ok) issue(c + 1);
    }
  }
  // every MMA of this CTA is complete once the last committed chunk's phase is
  if (last >= 0 && !tc::mbar_wait(&bars[last & 1], (uint32_t)((last >> 1) & 1))) ok = false;
  cp_async_wait<0>();
  ok = __syncthreads_and(ok) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int r = tl.row0 + warp * 32 + lane;
    for (int c0 = 0; c0 < tl.n_cols; c0 += 16) {
      uint32_t v[16];
      tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (r < R) {
        float* yr = Y + (long long)(r / seg) * seg_stride + r % seg;
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (c0 + j < tl.n_cols) yr[dsts[c0 + j] + tl.dst_off] = __uint_as_float(v[j]);
      }
    }
  } else if (tid == 0) {
    atomicExch(status, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NC));
}

constexpr int kXlSplit = 2;  // k ranges of the tensor-core wave -> local GEMM (measured: 2 beats 1, 3 and 4)

// L[ldst[col] + r] = sum over the k-range partials of column col (in order)
__global__ void __launch_bounds__(256) xl_reduce_kernel(int ncols, int R2, const long long* __restrict__ ldst,
                                                        const float* __restrict__ P, float* __restrict__ L) {
  pdl_begin();
  const long long total = (long long)ncols * R2;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total; o += (long long)gridDim.x * blockDim.x) {
    const int col = (int)(o / R2), r = (int)(o - (long long)col * R2);
    float v = P[o];
#pragma unroll
    for (int sp = 1; sp < kXlSplit; ++sp) v += P[(long long)sp * total + o];
    L[ldst[col] + r] = v;
  }
}

// M[parent] = sum of its children's partials, in child order
template <typename T>
__global__ void __launch_bounds__(256) shift_reduce_kernel(int E, const ShiftReduce* __restrict__ items,
                                                           const T* __restrict__ P, T* __restrict__ M) {
  pdl_begin();
  const int R = 2 * E;
  const ShiftReduce it = items[blockIdx.x];
  for (int o = threadIdx.x; o < kCh * R; o += blockDim.x) {
    T v = P[(size_t)it.first_slot * kCh * R + o];
    for (int j = 1; j < it.n_slots; ++j) v += P[(size_t)(it.first_slot + j) * kCh * R + o];
    M[(size_t)it.parent * kCh * R + o] = v;
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
  pdl_begin();
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
  // work of one far-field pass: columns (node, channel) of the M->X and
  // wave->local operators, translation entries, M2M / L2L columns
  FmmWork work;
  // chained far-field kernels launched as programmatic dependents
  bool pdl = true;
  // buffers a far-field plan shares among problems (see FmmPlan)
  using SharedBuf = std::shared_ptr<DevBuf>;
  SharedBuf tables_buf = std::make_shared<DevBuf>();  // one allocation holding every table
  DevBuf tables_buf_d;  // FP64 tables used only to tabulate operators of an FP32 problem
  Tables<double> tb_d{};
  Tables<float> tb_f{};
  DevBuf M, L, W;  // expansions and plane waves
  DevBuf p2m_items, xl_targets, xl_entries, leaf_items;
  int n_p2m = 0, n_leaf = 0;
  size_t smem_p2m = 0, smem_shift = 0, smem_m2x = 0, smem_prep = 0, smem_eval = 0, smem_op = 0, smem_xlb = 0;
  // operator form of multipole -> plane waves and accumulated waves -> local
  SharedBuf m2x_ops = std::make_shared<DevBuf>();  // [lg][2E][m2x_rp]
  SharedBuf xl_ops = std::make_shared<DevBuf>();   // [lg][12 NPM][xl_rp]
  int m2x_rp = 0, xl_rp = 0;
  DevBuf op_tiles, op_cols;
  DevBuf acc;      // [target row][channel][6 dirs][NPM] accumulated waves
  // FP32 engine: the same operators packed for the tensor cores (hi / lo
  // halves in the MMA's shared-memory layout), row tiles and k chunks
  bool tensor = false;
  SharedBuf m2x_tc = std::make_shared<DevBuf>(), xl_tc = std::make_shared<DevBuf>();
  int m2x_mt = 0, m2x_nc = 0, xl_mt = 0, xl_nc = 0;
  DevBuf tc_status;  // int[2]: [0] set by a tensor-core kernel whose wait timed out; [1] timeout test switch
  // split-K wave -> local: per level the columns' L offsets and the partials
  DevBuf xl_ldst, xl_partials;
  std::vector<int> xlr_first, xlr_count;
  std::vector<long long> xlr_pbase;
  DevBuf leaf_exp;  // per leaf: [2 groups][F, H0, H1, H2][EQ]
  DevBuf eval_items;
  DevBuf p2m_basis;   // [patch position][2 groups][E], geometry only
  DevBuf eval_basis;  // [eval item][2 groups][EQ][kEvalChunk], geometry only
  int n_eval = 0;
  // operator form of M2M / L2L and of the L2P preparation
  SharedBuf shift_ops = std::make_shared<DevBuf>();  // [op][k][r], op = ((kind*nlev + level)*2 + group)*8 + octant-1
  DevBuf shift_tiles, shift_cols, m2m_reduce, m2m_partials;
  std::vector<int> m2m_tfirst, m2m_tcount, m2m_rfirst, m2m_rcount;  // per child level
  std::vector<int> l2l_tfirst, l2l_tcount;                          // per parent level
  SharedBuf prep_rowptr = std::make_shared<DevBuf>(), prep_cols = std::make_shared<DevBuf>(),
            prep_vals = std::make_shared<DevBuf>();
  size_t smem_gemm = 0, smem_csr = 0;
  // per level: M2X tiles of the level's nodes, X2L targets on the level and
  // their conversion tiles; a stream per level runs them as soon as the
  // level's multipoles exist (events order them against the up and down
  // passes)
  std::vector<int> m2x_tfirst, m2x_tcount, xlt_first, xlt_count, xlc_tfirst, xlc_tcount;
  std::vector<cudaStream_t> lstreams;
  std::vector<cudaEvent_t> ev_m, ev_x;
  ~FmmState() {
    for (cudaEvent_t e : ev_m) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_x) cudaEventDestroy(e);
    for (cudaStream_t t : lstreams) cudaStreamDestroy(t);
  }
};

// The part of a far-field set-up that depends only on the FMM order, the
// screening constants, the cube edge, the number of levels and the
// precision: the device tables and the dense operators tabulated from them
// (M2M / L2L shifts, L2P preparation for every level, multipole -> waves
// and waves -> local, packed for the tensor cores in the FP32 engine).  A
// context keeps its few most recent plans; a problem built on it with the
// same key (a pose of a scan whose bounding cube is unchanged) adopts the
// plan instead of computing it, and holds it while it lives.
struct FmmPlan {
  int nt = 0, nlev = 0;
  double kappa = 0, beta0 = 0, edge = 0;
  bool fp64 = true;
  int np_max = 0, nl = 0;
  Tables<double> tb_d{};
  Tables<float> tb_f{};
  FmmState::SharedBuf tables_buf, shift_ops, prep_rowptr, prep_cols, prep_vals, m2x_ops, xl_ops, m2x_tc, xl_tc;
  int m2x_mt = 0, m2x_nc = 0, xl_mt = 0, xl_nc = 0;
  size_t smem_csr = 0;
  bool matches(const Problem& P, int levels) const {
    return nt == P.params.nterms && nlev == levels && kappa == P.params.kappa && beta0 == P.params.beta0 &&
           edge == P.params.cube_edge && fp64 == P.fp64;
  }
};

static std::shared_ptr<FmmPlan> find_fmm_plan(Problem& P, int levels) {
  Ctx* c = P.ctx;
  std::lock_guard<std::mutex> lk(c->plan_mu);
  for (size_t k = 0; k < c->fmm_plans.size(); ++k)
    if (c->fmm_plans[k]->matches(P, levels)) {
      std::shared_ptr<FmmPlan> p = c->fmm_plans[k];
      c->fmm_plans.erase(c->fmm_plans.begin() + k);
      c->fmm_plans.push_back(p);  // most recently used last
      return p;
    }
  return nullptr;
}

static void keep_fmm_plan(Problem& P, const FmmState& S) {
  auto p = std::make_shared<FmmPlan>();
  p->nt = S.nt;
  p->nlev = S.nlev;
  p->kappa = P.params.kappa;
  p->beta0 = P.params.beta0;
  p->edge = P.params.cube_edge;
  p->fp64 = S.fp64;
  p->np_max = S.np_max;
  p->nl = S.nl;
  if (S.fp64)
    p->tb_d = S.tb_d;  // an FP32 plan's FP64 tables were only used to tabulate its operators
  p->tb_f = S.tb_f;
  p->tables_buf = S.tables_buf;
  p->shift_ops = S.shift_ops;
  p->prep_rowptr = S.prep_rowptr;
  p->prep_cols = S.prep_cols;
  p->prep_vals = S.prep_vals;
  p->m2x_ops = S.m2x_ops;
  p->xl_ops = S.xl_ops;
  p->m2x_tc = S.m2x_tc;
  p->xl_tc = S.xl_tc;
  p->m2x_mt = S.m2x_mt;
  p->m2x_nc = S.m2x_nc;
  p->xl_mt = S.xl_mt;
  p->xl_nc = S.xl_nc;
  p->smem_csr = S.smem_csr;
  Ctx* c = P.ctx;
  std::lock_guard<std::mutex> lk(c->plan_mu);
  c->fmm_plans.push_back(p);
  while (c->fmm_plans.size() > Ctx::kFmmPlans) c->fmm_plans.erase(c->fmm_plans.begin());
}

void fmm_destroy(FmmState* s) { delete s; }

bool fmm_active(const Problem& P) { return P.tree.n_levels - 1 >= 2; }

FmmWork fmm_work(const Problem& P) { return P.fmm ? P.fmm->work : FmmWork{}; }

void fmm_check_waits(Problem& P) {
  FmmState* S = P.fmm.get();
  if (!S || !S->tc_status.get()) return;
  int flag = 0;
  BP_CUDA(cudaMemcpyAsync(&flag, S->tc_status.get(), sizeof(int), cudaMemcpyDeviceToHost, P.ctx->stream));
  BP_CUDA(cudaStreamSynchronize(P.ctx->stream));
  if (flag) {
    // reported once: the next matvec starts clean
    BP_CUDA(cudaMemsetAsync(S->tc_status.get(), 0, sizeof(int), P.ctx->stream));
    BP_CUDA(cudaStreamSynchronize(P.ctx->stream));
    throw TimeoutError("a tensor-core FMM kernel timed out waiting for its matrix multiplies");
  }
}

const int* fmm_status_dev(Problem& P) {
  FmmState* S = P.fmm.get();
  return S && S->tc_status.get() ? S->tc_status.as<int>() : nullptr;
}

void fmm_raise_if(Problem& P, int flag) {
  if (!flag) return;
  FmmState* S = P.fmm.get();
  BP_CUDA(cudaMemsetAsync(S->tc_status.get(), 0, sizeof(int), P.ctx->stream));
  BP_CUDA(cudaStreamSynchronize(P.ctx->stream));
  throw TimeoutError("a tensor-core FMM kernel timed out waiting for its matrix multiplies");
}

bool fmm_set_stall_test(Problem& P, bool on) {
  FmmState* S = P.fmm.get();
  if (!S || !S->tensor || !S->tc_status.get()) return false;
  const int v = on ? 1 : 0;
  BP_CUDA(cudaMemcpyAsync(S->tc_status.as<int>() + 1, &v, sizeof(int), cudaMemcpyHostToDevice, P.ctx->stream));
  BP_CUDA(cudaStreamSynchronize(P.ctx->stream));
  return true;
}

namespace {

template <typename T>
void fill_tables(FmmState& S, const Problem& P, Tables<T>& tb, DevBuf& buf, const GlobalTables& G,
                 const std::vector<LevelTables>& LT) {
  using C = typename C2T<T>::type;
  const int nt = S.nt, E = S.E, nlev = S.nlev;
  const double beta = std::max(P.params.kappa, P.params.beta0);
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
  std::vector<cplx> fexpe, fexpo, fexpback, xs, ys, tcomb;
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
    // translate_up/down_wave factor of every (up, a, b, c) offset combo:
    // up: zs[c] ys[b] xs[a] (conjugated factors for negative offsets),
    // down: zs[-c] with the conjugations reversed
    for (int combo = 0; combo < kCombos; ++combo) {
      const int up = combo / 343, a = (combo / 49) % 7 - 3, b = (combo / 7) % 7 - 3, c = combo % 7 - 3;
      for (int i = 0; i < npm; ++i) {
        if (i >= t.nexptotp) {
          tcomb.push_back(cplx(0));
          continue;
        }
        auto X = [&](int k) { return t.xs[(size_t)(k - 1) * t.nexptotp + i]; };
        auto Y = [&](int k) { return t.ys[(size_t)(k - 1) * t.nexptotp + i]; };
        auto Z = [&](int k) { return t.zs[(size_t)(k - 1) * t.nexptotp + i]; };
        cplx f;
        if (up) {
          f = cplx(c > 0 ? Z(c) : 1.0, 0.0);
          if (b > 0) f *= Y(b);
          else if (b < 0) f *= std::conj(Y(-b));
          if (a > 0) f *= X(a);
          else if (a < 0) f *= std::conj(X(-a));
        } else {
          f = cplx(c < 0 ? Z(-c) : 1.0, 0.0);
          if (b > 0) f *= std::conj(Y(b));
          else if (b < 0) f *= Y(-b);
          if (a > 0) f *= std::conj(X(a));
          else if (a < 0) f *= X(-a);
        }
        tcomb.push_back(f);
      }
    }
  }
  if (fexpe.empty()) fexpe.push_back(0);
  if (fexpo.empty()) fexpo.push_back(0);
  size_t o_np = putI(numphys), o_ne = putI(nexptot), o_nep = putI(nexptotp), o_sc = putT(scale),
         o_bs = putT(betascal), o_beta = putT(std::vector<double>{beta, P.params.beta0}), o_rl = putT(rlsc),
         o_fe = putC(fexpe), o_fo = putC(fexpo), o_fb = putC(fexpback), o_feo = putI(fe_off), o_foo = putI(fo_off),
         o_fbo = putI(fb_off), o_xs = putC(xs), o_ys = putC(ys), o_zs = putT(zs), o_mps = putT(mps),
         o_lcs = putT(lcs), o_tc = putC(tcomb);
  buf.alloc(P.ctx, blob.size());
  BP_CUDA(cudaMemcpyAsync(buf.get(), blob.data(), blob.size(), cudaMemcpyHostToDevice, P.ctx->stream));
  BP_CUDA(cudaStreamSynchronize(P.ctx->stream));
  unsigned char* base = buf.as<unsigned char>();
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
  tb.tcomb = reinterpret_cast<const C*>(base + o_tc);
  for (auto& t : LT)
    if (t.nexptot > 64) throw std::invalid_argument("FMM order with more than 64 Fourier modes is not supported");
}

}  // namespace


// Tabulates the operator form of M2M / L2L (one dense R x R matrix per
// kind, level, screening group and octant, R = 2E reals) and of the L2P
// preparation (one sparse matrix per leaf level) by applying the structured
// kernels to unit vectors.
// CSR of a dense operator stored by columns (D[b][rows]): one warp per row
// counts its nonzeros, then writes them in column order.
template <typename T>
__global__ void csr_count_kernel(const T* __restrict__ D, int nb, int rows, int* __restrict__ counts) {
  const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (r >= rows) return;
  int n = 0;
  for (int b = lane; b < nb; b += 32) n += D[(size_t)b * rows + r] != T(0);
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if (lane == 0) counts[r] = n;
}
template <typename T>
__global__ void csr_fill_kernel(const T* __restrict__ D, int nb, int rows, const int* __restrict__ rowptr,
                                int* __restrict__ cols, T* __restrict__ vals) {
  const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (r >= rows) return;
  int pos = rowptr[r];
  for (int b0 = 0; b0 < nb; b0 += 32) {
    const int b = b0 + lane;
    const T v = b < nb ? D[(size_t)b * rows + r] : T(0);
    const unsigned m = __ballot_sync(0xffffffffu, v != T(0));
    if (v != T(0)) {
      const int k = pos + __popc(m & ((1u << lane) - 1u));
      cols[k] = b;
      vals[k] = v;
    }
    pos += __popc(m);
  }
}

template <typename T>
static void build_operators(Problem& P, FmmState& S, const Tables<T>& tb) {
  using C = typename C2T<T>::type;
  Ctx* c = P.ctx;
  cudaStream_t st = c->stream;
  const int E = S.E, R = 2 * E, nlev = S.nlev, NT = S.nt;
  const int EQ = (NT + 3) * (NT + 4) / 2;
  // shifts: kind 0 = M2M (level = child level), kind 1 = L2L (level = parent level)
  const int n_ops = 2 * nlev * 2 * 8;
  S.shift_ops->alloc(c, sizeof(T) * (size_t)n_ops * R * ((R + 3) & ~3));
  shift_basis_kernel<T><<<n_ops * R, 64, S.smem_shift, st>>>(tb, nlev, S.shift_ops->as<T>());
  BP_LAUNCH_CHECK();
  // L2P preparation operator per level that holds leaves: tabulated on unit
  // inputs (dense columns [b][rows]) and compacted to CSR on the device, the
  // nonzeros of a row in column order
  const int nb = kCh * R, rows = 8 * 2 * EQ;
  // every level below the root may hold leaves of a problem that shares the
  // operators
  std::vector<int> levels_with_leaves(nlev, 1);
  levels_with_leaves[0] = 0;
  DevBuf Lb(c, sizeof(C) * (size_t)nb * kCh * E);
  prep_basis_inputs<T><<<nb, 128, 0, st>>>(E, nb, Lb.as<C>());
  BP_LAUNCH_CHECK();
  std::vector<DevBuf> Db(nlev);
  DevBuf counts(c, sizeof(int) * (size_t)nlev * rows);
  BP_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), st));
  std::vector<LeafItem> bi(nb);
  for (int b = 0; b < nb; ++b) bi[b] = LeafItem{b, 0, 0, 0, b, {0, 0, 0}};
  std::vector<DevBuf> d_bi(nlev);
  for (int lev = 0; lev < nlev; ++lev) {
    if (!levels_with_leaves[lev]) continue;
    for (int b = 0; b < nb; ++b) bi[b].level = lev;
    d_bi[lev] = upload(c, bi);
    Db[lev].alloc(c, sizeof(C) * (size_t)nb * 8 * EQ);
    l2p_prep_kernel<T><<<nb, 64, S.smem_prep, st>>>(tb, d_bi[lev].as<LeafItem>(), Lb.as<C>(), Db[lev].as<C>());
    BP_LAUNCH_CHECK();
    csr_count_kernel<T><<<(rows + 7) / 8, 256, 0, st>>>(Db[lev].as<T>(), nb, rows, counts.as<int>() + (size_t)lev * rows);
    BP_LAUNCH_CHECK();
  }
  std::vector<int> h_counts((size_t)nlev * rows);
  BP_CUDA(cudaMemcpyAsync(h_counts.data(), counts.get(), counts.bytes(), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  std::vector<int> rowptr((size_t)nlev * (rows + 1), 0);
  int nnz = 0;
  for (int lev = 0; lev < nlev; ++lev) {
    int* rp = rowptr.data() + (size_t)lev * (rows + 1);
    for (int r = 0; r < rows; ++r) {
      rp[r] = nnz;
      nnz += h_counts[(size_t)lev * rows + r];
    }
    rp[rows] = nnz;
  }
  *S.prep_rowptr = upload(c, rowptr);
  S.prep_cols->alloc(c, sizeof(int) * (size_t)std::max(1, nnz));
  S.prep_vals->alloc(c, sizeof(T) * (size_t)std::max(1, nnz));
  if (nnz == 0) {
    BP_CUDA(cudaMemsetAsync(S.prep_cols->get(), 0, sizeof(int), st));
    BP_CUDA(cudaMemsetAsync(S.prep_vals->get(), 0, sizeof(T), st));
  }
  for (int lev = 0; lev < nlev; ++lev) {
    if (!levels_with_leaves[lev]) continue;
    csr_fill_kernel<T><<<(rows + 7) / 8, 256, 0, st>>>(Db[lev].as<T>(), nb, rows,
                                                       S.prep_rowptr->as<int>() + (size_t)lev * (rows + 1),
                                                       S.prep_cols->as<int>(), S.prep_vals->as<T>());
    BP_LAUNCH_CHECK();
  }
  S.smem_csr = sizeof(T) * (size_t)kCh * R;
  BP_CUDA(cudaStreamSynchronize(st));
}

// M->X operator columns of one level from the tabulated waves of the unit
// multipoles: ops[lg][b][dir * 2 NPM + 2 i + re/im] = W[b][dir][ch0][i]
// (ch0 = 0 / 8 for the two screening groups); padding rows stay 0.
__global__ void m2x_columns_kernel(const double2* __restrict__ W, int R2, int NPM, int lev, int rp,
                                   double* __restrict__ ops) {
  const int total = 2 * R2 * 6 * NPM;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
    const int i = o % NPM, dir = (o / NPM) % 6, b = (o / (6 * NPM)) % R2, g = o / (6 * NPM * R2);
    const double2 w = W[(((size_t)b * 6 + dir) * kCh + (g ? 8 : 0)) * NPM + i];
    double* col = ops + ((size_t)(2 * (lev - 1) + g) * R2 + b) * rp + (size_t)dir * 2 * NPM + 2 * i;
    col[0] = w.x;
    col[1] = w.y;
  }
}

// ops[lg][k][row] (rows padded to RP) -> the tensor-core blocks
// [lg][row tile][k chunk][hi, lo][8 panels][128 rows][4] of op_gemm_tc_kernel;
// hi = the FP32 value with its 13 low mantissa bits cleared, lo = rest.
__global__ void pack_tensor_kernel(const double* __restrict__ ops, int nlg, int K, int RP, int R, int n_mt, int n_ch,
                                   float* __restrict__ out) {
  constexpr int kBlk = 2 * tc::kHalf / 4;  // floats per [hi, lo] block
  const long long total = (long long)nlg * n_mt * n_ch * (kBlk / 2);
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(o % (kBlk / 2));  // q * 512 + r * 4 + u
    const long long blk = o / (kBlk / 2);
    const int ch = (int)(blk % n_ch), mt = (int)((blk / n_ch) % n_mt), lg = (int)(blk / ((long long)n_ch * n_mt));
    const int q = e / (tc::kRows * 4), r = (e / 4) % tc::kRows, u = e % 4;
    const int row = mt * tc::kRows + r, k = ch * tc::kKC + 4 * q + u;
    float a = 0.f;
    if (row < R && k < K) a = (float)ops[((size_t)lg * K + k) * RP + row];
    const float h = __uint_as_float(__float_as_uint(a) & 0xFFFFE000u);
    float* b = out + blk * kBlk;
    b[e] = h;
    b[kBlk / 2 + e] = a - h;
  }
}

// The dense M->X and waves->local operators of every level, tabulated in
// FP64 on the device by applying the structured kernels to unit vectors, and
// left on the device: packed for the tensor cores (FP32 engine) or as they
// are (FP64 engine).
static void build_wave_operators(Problem& P, FmmState& S) {
  Ctx* c = P.ctx;
  cudaStream_t st = c->stream;
  const int E = S.E, R2 = 2 * E, NPM = S.np_max, KW = 12 * NPM, nlev = S.nlev, nlg = 2 * nlev;
  DevBuf m2x(c, sizeof(double) * (size_t)nlg * R2 * S.m2x_rp);
  BP_CUDA(cudaMemsetAsync(m2x.get(), 0, m2x.bytes(), st));
  {
    std::vector<double2> hm((size_t)R2 * kCh * E, make_double2(0.0, 0.0));
    for (int b = 0; b < R2; ++b)
      for (int ch = 0; ch < kCh; ++ch) {
        double2& v = hm[((size_t)b * kCh + ch) * E + b / 2];
        if (b & 1) v.y = 1.0;
        else v.x = 1.0;
      }
    DevBuf Mb = upload(c, hm);
    DevBuf Wb(c, sizeof(double2) * (size_t)R2 * 6 * kCh * NPM);
    std::vector<M2xItem> items((size_t)nlev * R2);
    for (int lev = 1; lev < nlev; ++lev)
      for (int b = 0; b < R2; ++b) items[(size_t)lev * R2 + b] = M2xItem{b, lev};
    DevBuf di = upload(c, items);
    for (int lev = 1; lev < nlev; ++lev) {
      BP_CUDA(cudaMemsetAsync(Wb.get(), 0, Wb.bytes(), st));
      m2x_kernel<double><<<R2 * (kCh / kM2xChannels), kM2xThreads, S.smem_m2x, st>>>(
          S.tb_d, di.as<M2xItem>() + (size_t)lev * R2, Mb.as<double2>(), Wb.as<double2>());
      BP_LAUNCH_CHECK();
      m2x_columns_kernel<<<128, 256, 0, st>>>(Wb.as<double2>(), R2, NPM, lev, S.m2x_rp, m2x.as<double>());
      BP_LAUNCH_CHECK();
    }
    BP_CUDA(cudaStreamSynchronize(st));  // the host staging vectors go out of scope
  }
  DevBuf xl(c, sizeof(double) * (size_t)nlg * KW * S.xl_rp);
  BP_CUDA(cudaMemsetAsync(xl.get(), 0, xl.bytes(), st));
  for (int pl = 0; pl + 1 < nlev; ++pl) {
    xl_convert_basis_kernel<double><<<2 * KW, kPairLanes, S.smem_xlb, st>>>(S.tb_d, pl, S.xl_rp, xl.as<double>());
    BP_LAUNCH_CHECK();
  }
  if (S.tensor) {
    auto pack = [&](const DevBuf& ops, int K, int RP, int R, int& n_mt, int& n_ch, DevBuf& out) {
      n_mt = (R + tc::kRows - 1) / tc::kRows;
      n_ch = (K + tc::kKC - 1) / tc::kKC;
      out.alloc(c, sizeof(float) * (size_t)nlg * n_mt * n_ch * (2 * tc::kHalf / 4));
      pack_tensor_kernel<<<4 * c->sm_count, 256, 0, st>>>(ops.as<double>(), nlg, K, RP, R, n_mt, n_ch,
                                                          out.as<float>());
      BP_LAUNCH_CHECK();
    };
    pack(m2x, R2, S.m2x_rp, KW, S.m2x_mt, S.m2x_nc, *S.m2x_tc);
    pack(xl, KW, S.xl_rp, R2, S.xl_mt, S.xl_nc, *S.xl_tc);
  } else {  // the FP64 engine (the FP32 engine always takes the tensor cores)
    *S.m2x_ops = std::move(m2x);
    *S.xl_ops = std::move(xl);
  }
  BP_CUDA(cudaStreamSynchronize(st));
}

// Builds the FMM schedule of a problem.  Only work that can reach a result
// is scheduled: X2L halves with at least one interaction, M2X of the nodes
// that are translation sources, M2M / P2M of the nodes whose multipoles feed
// one of those, L2L out of nodes whose locals can be non-zero.  Every local
// expansion that is read is written in the same matvec (X2L or L2L assign
// it) or is identically zero (set once here).
void fmm_setup(Problem& P) {
  auto S = new FmmState();
  P.fmm.reset(S);
  const TreeInfo& T = P.tree;
  S->nt = P.params.nterms;
  S->E = (S->nt + 1) * (S->nt + 2) / 2;
  S->nlev = T.n_levels;
  S->fp64 = P.fp64;
  const std::shared_ptr<FmmPlan> plan = find_fmm_plan(P, S->nlev);
  if (plan) {
    S->tables_buf = plan->tables_buf;
    S->tb_d = plan->tb_d;
    S->tb_f = plan->tb_f;
    S->np_max = plan->np_max;
    S->nl = plan->nl;
  } else {
    // FP64 tables always: they tabulate the dense operators of both engines
    // host tables (FP64) once; both engines' device copies are made from them
    GlobalTables G;
    G.build(S->nt);
    std::vector<LevelTables> LT(2 * S->nlev);
    const double beta = std::max(P.params.kappa, P.params.beta0);
    for (int l = 0; l < S->nlev; ++l) {
      LT[2 * l].build(S->nt, beta, l, P.params.cube_edge);
      LT[2 * l + 1].build(S->nt, P.params.beta0, l, P.params.cube_edge);
    }
    fill_tables<double>(*S, P, S->tb_d, S->fp64 ? *S->tables_buf : S->tables_buf_d, G, LT);
    if (!S->fp64) fill_tables<float>(*S, P, S->tb_f, *S->tables_buf, G, LT);
  }
  if (S->np_max > kPairLanes) throw std::invalid_argument("FMM order too large for the plane-wave thread layout");
  const int nn = (int)T.nodes.size();
  const size_t celem = S->fp64 ? sizeof(double2) : sizeof(float2);
  const size_t exp_bytes = (size_t)nn * kCh * S->E * celem;
  S->M.alloc(P.ctx, exp_bytes);
  S->L.alloc(P.ctx, exp_bytes);
  BP_CUDA(cudaMemsetAsync(S->L.get(), 0, exp_bytes, P.ctx->stream));
  S->W.alloc(P.ctx, (size_t)nn * 6 * kCh * S->np_max * celem);
  BP_CUDA(cudaMemsetAsync(S->W.get(), 0, S->W.bytes(), P.ctx->stream));
  const int nlev = S->nlev;
  auto flags = [&](int k) { return T.nodes[k].flags; };
  auto cnt = [&](int k) { return T.nodes[k].content_count; };
  auto octant = [&](int k) { return 1 + (T.nodes[k].ix & 1) + 2 * (T.nodes[k].iy & 1) + 4 * (T.nodes[k].iz & 1); };
  // X2L targets: non-shadow children of parents that are neither leaf nor
  // shadow, with at least one interaction; entries sorted by direction
  const auto table = interaction_table();
  std::vector<std::vector<int>> by_target_dir(8 * 6);
  for (int q = 0; q < (int)table.size(); ++q) by_target_dir[table[q].targ * 6 + table[q].dir].push_back(q);
  std::vector<std::vector<XlTarget>> xlt_lev(nlev);
  std::vector<XlEntry> xle;
  std::vector<char> is_source(nn, 0), written(nn, 0);
  for (int k = 0; k < nn; ++k) {
    const TreeNode& nd = T.nodes[k];
    if (nd.level >= nlev - 1) continue;
    if ((nd.flags & TREE_LEAF) || (nd.flags & TREE_SHADOW)) continue;
    for (int t = 0; t < 8; ++t) {
      const int ck = nd.children[t];
      if (ck < 0 || (flags(ck) & TREE_SHADOW)) continue;
      XlTarget tg{ck, 0, (int)xle.size(), 0, {0, 0, 0, 0, 0, 0, 0}};
      for (int dir = 0; dir < 6; ++dir) {
        tg.dir_start[dir] = (int)xle.size() - tg.first_entry;
        for (int q : by_target_dir[t * 6 + dir]) {
          const RawInteraction& r = table[q];
          const int nbk = nd.neighbours[r.nb];
          if (nbk < 0 || cnt(nbk) == 0) continue;
          const int sk = T.nodes[nbk].children[r.src];
          if (sk < 0 || cnt(sk) == 0) continue;
          int a, b, c;
          switch (r.dir) {
            case 0: case 1: a = r.dx; b = r.dy; c = r.dz; break;
            case 2: case 3: a = r.dz; b = r.dx; c = r.dy; break;
            default: a = -r.dz; b = r.dy; c = r.dx; break;
          }
          const int up = r.dir % 2 == 0 ? 1 : 0;
          XlEntry e;
          e.src = sk;
          e.combo = (short)(up * 343 + (a + 3) * 49 + (b + 3) * 7 + (c + 3));
          e.dir = (signed char)r.dir;
          e.pad = 0;
          xle.push_back(e);
          is_source[sk] = 1;
        }
      }
      tg.n_entries = (int)xle.size() - tg.first_entry;
      tg.dir_start[6] = tg.n_entries;
      if (tg.n_entries == 0) continue;
      written[ck] = 1;
      xlt_lev[nd.level + 1].push_back(tg);
    }
  }
  // multipoles needed: translation sources and every node below one
  // (nodes are stored level by level, parents first)
  std::vector<char> mneed(nn, 0), lnz(nn, 0);
  for (int k = 0; k < nn; ++k) {
    const int p = T.nodes[k].parent;
    mneed[k] = is_source[k] || (p >= 0 && mneed[p]);
    lnz[k] = written[k] || (p >= 0 && lnz[p]);
  }
  // P2M items
  std::vector<P2mItem> p2m;
  int p2m_rows = 0;
  for (int k = 0; k < nn; ++k) {
    if ((flags(k) & TREE_HAS_CHILDREN) || cnt(k) == 0 || !mneed[k]) continue;
    P2mItem it{k, T.nodes[k].level, (int)T.nodes[k].content_start, cnt(k), p2m_rows, {0, 0, 0}};
    for (int d = 0; d < 3; ++d) it.c[d] = T.nodes[k].centre[d];
    p2m.push_back(it);
    p2m_rows += cnt(k);
  }
  auto op_base = [&](int kind, int level, int oct) { return ((kind * nlev + level) * 2) * 8 + oct - 1; };
  // M2M / L2L tiles: columns bucketed by (octant, screening group) so that
  // a tile shares one operator; M2M columns write partial slots
  std::vector<ShiftTile> tiles;
  std::vector<ShiftCol> tcols;
  std::vector<ShiftReduce> reds;
  auto add_bucket = [&](int op, const std::vector<ShiftCol>& bucket) {
    for (size_t b0 = 0; b0 < bucket.size(); b0 += kTileCols) {
      ShiftTile t{op, (int)tcols.size(), (int)std::min<size_t>(kTileCols, bucket.size() - b0)};
      tcols.insert(tcols.end(), bucket.begin() + b0, bucket.begin() + b0 + t.n_cols);
      tiles.push_back(t);
    }
  };
  S->m2m_tfirst.assign(nlev, 0);
  S->m2m_tcount.assign(nlev, 0);
  S->m2m_rfirst.assign(nlev, 0);
  S->m2m_rcount.assign(nlev, 0);
  int n_slots = 0;
  for (int lev = nlev - 1; lev >= 1; --lev) {
    std::vector<std::vector<ShiftCol>> bucket(16);  // [group][octant-1]
    S->m2m_rfirst[lev] = (int)reds.size();
    for (int k = T.level_start[lev - 1]; k < T.level_start[lev]; ++k) {
      if (!(flags(k) & TREE_HAS_CHILDREN) || cnt(k) == 0 || !mneed[k]) continue;
      ShiftReduce r{k, n_slots, 0};
      for (int c = 0; c < 8; ++c) {
        const int ck = T.nodes[k].children[c];
        if (ck < 0 || cnt(ck) == 0) continue;
        const int oct = octant(ck), slot = n_slots + r.n_slots++;
        for (int ch = 0; ch < kCh; ++ch) bucket[(ch >= 8 ? 8 : 0) + oct - 1].push_back({ck, slot, ch, 0});
      }
      if (r.n_slots) {
        reds.push_back(r);
        n_slots += r.n_slots;
      }
    }
    S->m2m_rcount[lev] = (int)reds.size() - S->m2m_rfirst[lev];
    S->m2m_tfirst[lev] = (int)tiles.size();
    for (int b = 0; b < 16; ++b) add_bucket(op_base(0, lev, b % 8 + 1) + (b >= 8 ? 8 : 0), bucket[b]);
    S->m2m_tcount[lev] = (int)tiles.size() - S->m2m_tfirst[lev];
  }
  // translation sources per level (their multipoles become plane waves)
  std::vector<std::vector<int>> src_lev(nlev);
  for (int k = 0; k < nn; ++k)
    if (is_source[k]) src_lev[T.nodes[k].level].push_back(k);
  // L2L per parent level, top-down: child (= or +=) shift(parent)
  S->l2l_tfirst.assign(nlev, 0);
  S->l2l_tcount.assign(nlev, 0);
  for (int lev = 0; lev < nlev - 1; ++lev) {
    std::vector<std::vector<ShiftCol>> bucket(16);
    for (int k = T.level_start[lev]; k < T.level_start[lev + 1]; ++k) {
      if (!(flags(k) & TREE_HAS_CHILDREN) || (flags(k) & TREE_LEAF) || !lnz[k]) continue;
      for (int c = 0; c < 8; ++c) {
        const int ck = T.nodes[k].children[c];
        if (ck < 0 || cnt(ck) == 0 || (flags(ck) & TREE_SHADOW)) continue;
        for (int ch = 0; ch < kCh; ++ch) bucket[(ch >= 8 ? 8 : 0) + c].push_back({k, ck, ch, written[ck] ? 1 : 0});
      }
    }
    S->l2l_tfirst[lev] = (int)tiles.size();
    for (int b = 0; b < 16; ++b) add_bucket(op_base(1, lev, b % 8 + 1) + (b >= 8 ? 8 : 0), bucket[b]);
    S->l2l_tcount[lev] = (int)tiles.size() - S->l2l_tfirst[lev];
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
  // operator GEMM tiles: M2X columns (source node, channel) per (level,
  // group) into W; X->L columns (target, channel) per (level, group) from the
  // ACC scratch into L
  const int NPM = S->np_max, R2 = 2 * S->E, KW = 12 * NPM;
  S->m2x_rp = (KW + kOpRows - 1) / kOpRows * kOpRows;
  S->xl_rp = (R2 + kOpRows - 1) / kOpRows * kOpRows;
  std::vector<GemmTile> otiles;
  std::vector<GemmCol> ocols;
  // FP32 engine: 128 x 128 tensor-core tiles over the valid rows; FP64
  // engine: 112 x 32 SIMT tiles over the padded rows
  S->tensor = !S->fp64;
  const int tile_rows = S->tensor ? tc::kRows : kOpRows;
  S->m2x_mt = (KW + tc::kRows - 1) / tc::kRows;
  S->m2x_nc = (R2 + tc::kKC - 1) / tc::kKC;
  S->xl_mt = (R2 + tc::kRows - 1) / tc::kRows;
  S->xl_nc = (KW + tc::kKC - 1) / tc::kKC;
  // k chunks [kc0, kc0 + nkc) of every tile; dst_off shifts its outputs
  auto add_cols = [&](int op, int rows_pad, const std::vector<GemmCol>& cl, int tile_cols, int kc0, int nkc,
                      long long dst_off) {
    for (size_t c0 = 0; c0 < cl.size(); c0 += tile_cols) {
      const int n = (int)std::min<size_t>(tile_cols, cl.size() - c0);
      const int first = (int)ocols.size();
      ocols.insert(ocols.end(), cl.begin() + c0, cl.begin() + c0 + n);
      for (int row0 = 0; row0 < rows_pad; row0 += tile_rows) otiles.push_back({op, first, n, row0, kc0, nkc, dst_off});
    }
  };
  // wave -> local on the tensor cores: K split into kXlSplit ranges, each
  // tile writing a partial; xl_reduce_kernel sums the partials into L
  const int xl_per = (S->xl_nc + kXlSplit - 1) / kXlSplit;
  std::vector<long long> xl_ldst;
  long long xl_part = 0;
  S->xlr_first.assign(nlev, 0);
  S->xlr_count.assign(nlev, 0);
  S->xlr_pbase.assign(nlev, 0);
  S->m2x_tfirst.assign(nlev, 0);
  S->m2x_tcount.assign(nlev, 0);
  S->xlt_first.assign(nlev, 0);
  S->xlt_count.assign(nlev, 0);
  S->xlc_tfirst.assign(nlev, 0);
  S->xlc_tcount.assign(nlev, 0);
  std::vector<XlTarget> xlt;
  for (int lev = 1; lev < nlev; ++lev) {
    S->m2x_tfirst[lev] = (int)otiles.size();
    for (int g = 0; g < 2; ++g) {
      std::vector<GemmCol> cl;
      for (int k : src_lev[lev])
        for (int ch = g ? 8 : 0; ch < (g ? kCh : 8); ++ch)
          cl.push_back({((long long)k * kCh + ch) * R2, ((long long)k * 6 * kCh + ch) * 2 * NPM});
      add_cols(2 * (lev - 1) + g, S->tensor ? KW : S->m2x_rp, cl, S->tensor ? tc::kColsM2x : kOpCols, 0, S->m2x_nc, 0);
    }
    S->m2x_tcount[lev] = (int)otiles.size() - S->m2x_tfirst[lev];
    S->xlt_first[lev] = (int)xlt.size();
    for (XlTarget tg : xlt_lev[lev]) {
      tg.acc_row = (int)xlt.size();
      xlt.push_back(tg);
    }
    S->xlt_count[lev] = (int)xlt.size() - S->xlt_first[lev];
    S->xlc_tfirst[lev] = (int)otiles.size();
    S->xlr_first[lev] = (int)xl_ldst.size();
    S->xlr_pbase[lev] = xl_part;
    const long long ncl = (long long)S->xlt_count[lev] * kCh;  // columns of this level
    for (int g = 0; g < 2; ++g) {
      std::vector<GemmCol> cl;
      for (int q = S->xlt_first[lev]; q < S->xlt_first[lev] + S->xlt_count[lev]; ++q)
        for (int ch = g ? 8 : 0; ch < (g ? kCh : 8); ++ch) {
          GemmCol col{((long long)xlt[q].acc_row * kCh + ch) * KW, ((long long)xlt[q].node * kCh + ch) * R2};
          if (S->tensor) {  // output goes to the column's partial slot
            xl_ldst.push_back(col.dst);
            col.dst = (long long)(xl_ldst.size() - 1 - S->xlr_first[lev]) * R2;
          }
          cl.push_back(col);
        }
      if (!S->tensor) {
        add_cols(2 * (lev - 1) + g, S->xl_rp, cl, kOpCols, 0, 0, 0);
        continue;
      }
      for (int sp = 0; sp < kXlSplit; ++sp) {
        const int kc0 = sp * xl_per, nkc = std::min(xl_per, S->xl_nc - kc0);
        if (nkc > 0) add_cols(2 * (lev - 1) + g, R2, cl, tc::kColsXl, kc0, nkc, xl_part + sp * ncl * R2);
      }
    }
    S->xlc_tcount[lev] = (int)otiles.size() - S->xlc_tfirst[lev];
    S->xlr_count[lev] = (int)xl_ldst.size() - S->xlr_first[lev];
    if (S->tensor) xl_part += (long long)kXlSplit * ncl * R2;
  }
  {
    long long m2x = 0, x2l = 0;
    for (int lev = 1; lev < nlev; ++lev) {
      m2x += (long long)src_lev[lev].size() * kCh;
      x2l += (long long)S->xlt_count[lev] * kCh;
    }
    S->work.m2x_cols = m2x;
    S->work.x2l_cols = x2l;
    S->work.xl_entries = (long long)xle.size();
    S->work.shift_cols = (long long)tcols.size();
    S->work.plane_waves = S->np_max;
    S->work.coefficients = S->E;
  }
  S->op_tiles = upload(c, otiles);
  S->op_cols = upload(c, ocols);
  S->xl_targets = upload(c, xlt);
  S->xl_entries = upload(c, xle);
  S->acc.alloc(c, celem * kCh * 6 * (size_t)NPM * std::max<size_t>(1, xlt.size()));
  if (S->tensor) {
    S->xl_ldst = upload(c, xl_ldst);
    S->xl_partials.alloc(c, sizeof(float) * (size_t)std::max<long long>(1, xl_part));
  }
  // priorities: the upward chain (M2M), L2L and L2P on the FMM stream are the
  // critical path and keep the highest priority; the coarsest level with
  // interactions feeds the downward chain first, so each deeper level's
  // stream (M2X + X2L, not needed until later) is one step lower
  int prio_lo = 0, prio_hi = 0;
  BP_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  int top_x = nlev;
  for (int lev = 0; lev < nlev; ++lev)
    if (S->m2x_tcount[lev] > 0 || S->xlt_count[lev] > 0) {
      top_x = lev;
      break;
    }
  S->lstreams.assign(nlev, nullptr);
  S->ev_m.assign(nlev, nullptr);
  S->ev_x.assign(nlev, nullptr);
  for (int lev = 0; lev < nlev; ++lev) {
    const int prio = std::min(prio_lo, prio_hi + std::max(0, lev - top_x));
    BP_CUDA(cudaStreamCreateWithPriority(&S->lstreams[lev], cudaStreamNonBlocking, prio));
    BP_CUDA(cudaEventCreateWithFlags(&S->ev_m[lev], cudaEventDisableTiming));
    BP_CUDA(cudaEventCreateWithFlags(&S->ev_x[lev], cudaEventDisableTiming));
  }
  S->shift_tiles = upload(c, tiles);
  S->shift_cols = upload(c, tcols);
  S->m2m_reduce = upload(c, reds);
  S->m2m_partials.alloc(c, celem * kCh * (size_t)S->E * std::max(1, n_slots));
  S->leaf_items = upload(c, leaves);
  S->n_leaf = (int)leaves.size();
  S->eval_items = upload(c, evals);
  S->n_eval = (int)evals.size();
  const int E = S->E, NT = S->nt;
  if (E > kPairLanes || ((2 * E + 3) & ~3) > 112) throw std::invalid_argument("FMM order above 9 is not supported");
  S->smem_shift = 4 * celem * E;
  S->smem_p2m = celem * (size_t)kP2mChunk * 2 * E;
  S->smem_gemm = (S->fp64 ? 8 : 4) * (size_t)(2 * E) * (((2 * E + 3) & ~3) + kTileCols);
  S->smem_m2x = sizeof(double2) * (size_t)(4 * kM2xChannels * E + 6 * kM2xChannels * 64);  // FP64 tabulation
  S->smem_xlb = sizeof(double2) * (size_t)(6 * S->np_max + 6 * 64);
  S->smem_op = (S->fp64 ? 8 : 4) * (size_t)2 * (S->fp64 ? OpChunk<double>::value : OpChunk<float>::value) *
               (kOpRows + kOpCols);
  const int EQ = (NT + 3) * (NT + 4) / 2;
  S->smem_prep = celem * 2 * 24 * (size_t)EQ;
  S->smem_eval = celem * 8 * (size_t)EQ + (S->fp64 ? 8 : 4) * (size_t)16 * kEvalChunk +
                 (S->fp64 ? 0 : celem * 2 * (size_t)EQ * kEvalChunk);
  S->leaf_exp.alloc(P.ctx, celem * 8 * (size_t)EQ * std::max(1, S->n_leaf));
  S->p2m_basis.alloc(P.ctx, celem * 2 * (size_t)E * std::max(1, p2m_rows));
  S->eval_basis.alloc(P.ctx, celem * 2 * (size_t)EQ * kEvalChunk * std::max(1, S->n_eval));
  if (S->smem_op > 227 * 1024 || S->smem_prep > 227 * 1024 || S->smem_m2x > 227 * 1024 ||
      S->smem_gemm > 227 * 1024)
    throw std::invalid_argument("FMM order too large for the shared-memory layout");
  if (S->fp64) {
    ensure_dynamic_smem((const void*)op_gemm_kernel<double>, S->smem_op);
    ensure_dynamic_smem((const void*)shift_gemm_kernel<double>, S->smem_gemm);
    ensure_dynamic_smem((const void*)l2p_prep_kernel<double>, S->smem_prep);
    ensure_dynamic_smem((const void*)l2p_eval_kernel<double>, S->smem_eval);
    ensure_dynamic_smem((const void*)p2m_kernel<double>, S->smem_p2m);
  } else {
    ensure_dynamic_smem((const void*)op_gemm_kernel<float>, S->smem_op);
    ensure_dynamic_smem((const void*)shift_gemm_kernel<float>, S->smem_gemm);
    ensure_dynamic_smem((const void*)l2p_prep_kernel<float>, S->smem_prep);
    ensure_dynamic_smem((const void*)l2p_eval_kernel<float>, S->smem_eval);
    ensure_dynamic_smem((const void*)p2m_kernel<float>, S->smem_p2m);
  }
  ensure_dynamic_smem((const void*)m2x_kernel<double>, S->smem_m2x);
  if (S->tensor) {
    ensure_dynamic_smem((const void*)op_gemm_tc_kernel<tc::kColsM2x>, tc::smem_bytes(tc::kColsM2x));
    ensure_dynamic_smem((const void*)op_gemm_tc_kernel<tc::kColsXl>, tc::smem_bytes(tc::kColsXl));
  }
  S->tc_status.alloc(c, 2 * sizeof(int));
  BP_CUDA(cudaMemsetAsync(S->tc_status.get(), 0, 2 * sizeof(int), c->stream));
  // device copy of the tree contents (node-major)
  P.fmm_contents = upload(c, T.contents);
  BP_CUDA(cudaStreamSynchronize(c->stream));
  if (plan) {
    S->shift_ops = plan->shift_ops;
    S->prep_rowptr = plan->prep_rowptr;
    S->prep_cols = plan->prep_cols;
    S->prep_vals = plan->prep_vals;
    S->m2x_ops = plan->m2x_ops;
    S->xl_ops = plan->xl_ops;
    S->m2x_tc = plan->m2x_tc;
    S->xl_tc = plan->xl_tc;
    S->m2x_mt = plan->m2x_mt;
    S->m2x_nc = plan->m2x_nc;
    S->xl_mt = plan->xl_mt;
    S->xl_nc = plan->xl_nc;
    S->smem_csr = plan->smem_csr;
  } else {
    if (S->fp64)
      build_operators<double>(P, *S, S->tb_d);
    else
      build_operators<float>(P, *S, S->tb_f);
    build_wave_operators(P, *S);
    S->tables_buf_d.reset();  // the FP64 copy of an FP32 problem's tables is no longer needed
    keep_fmm_plan(P, *S);
  }
  // geometry-only bases of P2M and of the L2P evaluation
  const double* cen = P.d_centroid.as<double>();
  if (S->fp64) {
    if (S->n_p2m)
      p2m_basis_kernel<double><<<S->n_p2m, 64, 0, c->stream>>>(S->tb_d, S->p2m_items.as<P2mItem>(),
                                                               P.fmm_contents.as<int32_t>(), cen,
                                                               S->p2m_basis.as<double2>());
    if (S->n_eval)
      l2p_basis_kernel<double><<<S->n_eval, kEvalChunk, 0, c->stream>>>(S->tb_d, S->eval_items.as<LeafItem>(),
                                                                         P.fmm_contents.as<int32_t>(), cen,
                                                                         S->eval_basis.as<double2>());
  } else {
    if (S->n_p2m)
      p2m_basis_kernel<float><<<S->n_p2m, 64, 0, c->stream>>>(S->tb_f, S->p2m_items.as<P2mItem>(),
                                                              P.fmm_contents.as<int32_t>(), cen,
                                                              S->p2m_basis.as<float2>());
    if (S->n_eval)
      l2p_basis_kernel<float><<<S->n_eval, kEvalChunk, 0, c->stream>>>(S->tb_f, S->eval_items.as<LeafItem>(),
                                                                        P.fmm_contents.as<int32_t>(), cen,
                                                                        S->eval_basis.as<float2>());
  }
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(c->stream));
}

// One FMM pass.  With st == nullptr the levels overlap: the upward chain
// (P2M, M2M level by level) and the downward chain (L2L, L2P) run on the
// FMM stream, and each level's M2X + X2L runs on its own stream as soon as
// that level's multipoles are complete; L2L into a level waits for the
// level's X2L.  With st != nullptr (stage profiling) everything runs in
// order on one stream.
// One operator GEMM launch over tiles [first, first + count): tcgen05 for the
// FP32 engine, the SIMT kernel for the FP64 engine.
// A kernel launch on stream q; with pdl set, as a programmatic dependent of
// the kernel launched just before it on q (which it follows with no event
// wait in between): it may start while that kernel's last CTAs run and
// waits for it in pdl_begin.
template <typename... KArgs, typename... Args>
static void launch_k(bool pdl, void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t q,
                     Args... args) {
  if (!pdl) {
    kernel<<<grid, block, smem, q>>>(args...);
    BP_LAUNCH_CHECK();
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = q;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BP_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
}

template <typename T>
static void launch_op_gemm(FmmState& S, int first, int count, const T* simt_ops, const float* tc_ops, int n_mt,
                           int n_ch, int K, int RP, int R, int seg, long long seg_stride, const T* X, T* Y,
                           cudaStream_t q, int tc_cols, bool pdl) {
  if constexpr (std::is_same<T, float>::value) {
    if (S.tensor) {
      if (tc_cols == tc::kColsM2x)
        launch_k(pdl, op_gemm_tc_kernel<tc::kColsM2x>, count, tc::kThreads, tc::smem_bytes(tc::kColsM2x), q,
                 S.op_tiles.as<GemmTile>() + first, S.op_cols.as<GemmCol>(), tc_ops, n_mt, n_ch, K, R, seg, seg_stride,
                 X, Y, S.tc_status.as<int>());
      else
        launch_k(pdl, op_gemm_tc_kernel<tc::kColsXl>, count, tc::kThreads, tc::smem_bytes(tc::kColsXl), q,
                 S.op_tiles.as<GemmTile>() + first, S.op_cols.as<GemmCol>(), tc_ops, n_mt, n_ch, K, R, seg, seg_stride,
                 X, Y, S.tc_status.as<int>());
      return;
    }
  }
  launch_k(pdl, op_gemm_kernel<T>, count, kOpThreads, S.smem_op, q, S.op_tiles.as<GemmTile>() + first,
           S.op_cols.as<GemmCol>(), simt_ops, K, RP, R, seg, seg_stride, X, Y);
}

template <typename T>
static void run_fmm(Problem& P, FmmState& S, const Tables<T>& tb, const double* x, double* y, StageTimes* st,
                    cudaStream_t s) {
  using C = typename C2T<T>::type;
  C* M = S.M.as<C>();
  C* Lx = S.L.as<C>();
  C* W = S.W.as<C>();
  const int32_t* contents = P.fmm_contents.as<int32_t>();
  const bool overlap = st == nullptr;
  auto begin = [&](int stage, cudaStream_t q) {
    if (st) st->begin(stage, q);
  };
  auto end = [&](int launches) {
    if (st) st->end(launches);
  };
  if (S.n_leaf == 0) throw std::runtime_error("inconsistent FMM schedule (no leaves)");
  const int nlev = S.nlev;
  const int NPM = S.np_max, KW = 12 * NPM, R2 = 2 * S.E;
  auto has_x = [&](int lev) { return S.m2x_tcount[lev] > 0 || S.xlt_count[lev] > 0; };
  // multipole -> plane waves, translations, accumulated waves -> locals of
  // one level on stream q
  // programmatic dependent launches only inside a chain of kernels on one
  // stream: not for the first kernel after an event wait, and not when the
  // stages are timed one by one
  const bool pdl_ok = overlap && S.pdl;
  auto level_x = [&](int lev, cudaStream_t q) {
    bool chained = false;  // the previous operation on q is a kernel of this chain
    if (S.m2x_tcount[lev]) {
      begin(3, q);
      launch_op_gemm<T>(S, S.m2x_tfirst[lev], S.m2x_tcount[lev], S.m2x_ops->as<T>(), S.m2x_tc->as<float>(), S.m2x_mt,
                        S.m2x_nc, R2, S.m2x_rp, KW, 2 * NPM, (long long)kCh * 2 * NPM,
                        reinterpret_cast<const T*>(M), reinterpret_cast<T*>(W), q, tc::kColsM2x, false);
      end(1);
      chained = true;
    }
    if (S.xlt_count[lev]) {
      begin(4, q);
      const int nb = S.xlt_count[lev] * (kCh / kXlChannels);
      launch_k(pdl_ok && chained, xl_translate_kernel<T>, nb, kXlDirThreads, 0, q, tb, lev - 1,
               S.xl_targets.as<XlTarget>() + S.xlt_first[lev], S.xlt_count[lev], S.xl_entries.as<XlEntry>(),
               (const C*)W, S.acc.as<C>());
      if (S.tensor) {  // k-range partials, then their fixed-order sum into L
        launch_op_gemm<T>(S, S.xlc_tfirst[lev], S.xlc_tcount[lev], S.xl_ops->as<T>(), S.xl_tc->as<float>(), S.xl_mt,
                          S.xl_nc, KW, S.xl_rp, R2, R2, 0LL, reinterpret_cast<const T*>(S.acc.as<C>()),
                          reinterpret_cast<T*>(S.xl_partials.as<float>()), q, tc::kColsXl, pdl_ok);
        const long long total = (long long)S.xlr_count[lev] * R2;
        const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
        launch_k(pdl_ok, xl_reduce_kernel, grid, 256, 0, q, S.xlr_count[lev], R2,
                 S.xl_ldst.as<long long>() + S.xlr_first[lev], (const float*)(S.xl_partials.as<float>() + S.xlr_pbase[lev]),
                 reinterpret_cast<float*>(Lx));
        end(3);
      } else {
        launch_op_gemm<T>(S, S.xlc_tfirst[lev], S.xlc_tcount[lev], S.xl_ops->as<T>(), S.xl_tc->as<float>(), S.xl_mt,
                          S.xl_nc, KW, S.xl_rp, R2, R2, 0LL, reinterpret_cast<const T*>(S.acc.as<C>()),
                          reinterpret_cast<T*>(Lx), q, tc::kColsXl, pdl_ok);
        end(2);
      }
    }
  };
  auto fork_x = [&](int lev) {
    if (!has_x(lev)) return;
    if (!overlap) {
      level_x(lev, s);
      return;
    }
    BP_CUDA(cudaEventRecord(S.ev_m[lev], s));
    BP_CUDA(cudaStreamWaitEvent(S.lstreams[lev], S.ev_m[lev], 0));
    level_x(lev, S.lstreams[lev]);
    BP_CUDA(cudaEventRecord(S.ev_x[lev], S.lstreams[lev]));
  };
  auto join_x = [&](int lev) {
    if (overlap && has_x(lev)) BP_CUDA(cudaStreamWaitEvent(s, S.ev_x[lev], 0));
  };
  // upward pass
  begin(1, s);
  int l_p2m = 0;
  if (S.n_p2m) {
    p2m_kernel<T><<<S.n_p2m, 128, S.smem_p2m, s>>>(S.p2m_items.as<P2mItem>(), S.E, contents, P.d_area.as<double>(),
                                          P.d_normal.as<double>(), P.d_eps.as<double>(), x, P.n,
                                          S.p2m_basis.as<C>(), M);
    BP_LAUNCH_CHECK();
    ++l_p2m;
  }
  end(l_p2m);
  T* Mr = reinterpret_cast<T*>(M);
  T* Pr = S.m2m_partials.as<T>();
  bool chained = l_p2m > 0;  // the previous operation on s is a kernel of this chain
  for (int lev = nlev - 1; lev >= 0; --lev) {
    // multipoles of level lev are complete once its children's are shifted in
    if (lev + 1 < nlev && S.m2m_tcount[lev + 1]) {
      begin(2, s);
      launch_k(pdl_ok && chained, shift_gemm_kernel<T>, S.m2m_tcount[lev + 1], kGemmThreads, S.smem_gemm, s, S.E,
               (const ShiftTile*)(S.shift_tiles.as<ShiftTile>() + S.m2m_tfirst[lev + 1]),
               (const ShiftCol*)S.shift_cols.as<ShiftCol>(), (const T*)S.shift_ops->as<T>(), (const T*)Mr, Pr);
      launch_k(pdl_ok, shift_reduce_kernel<T>, S.m2m_rcount[lev + 1], 256, 0, s, S.E,
               (const ShiftReduce*)(S.m2m_reduce.as<ShiftReduce>() + S.m2m_rfirst[lev + 1]), (const T*)Pr, Mr);
      end(2);
      chained = true;
    }
    fork_x(lev);  // an event record on s: later kernels on s still follow a kernel
  }
  // downward pass: locals of level lev + 1 = X2L result (+) L2L of level lev
  for (int lev = 0; lev < nlev - 1; ++lev) {
    if (!S.l2l_tcount[lev]) continue;
    join_x(lev);
    join_x(lev + 1);
    begin(6, s);
    shift_gemm_kernel<T><<<S.l2l_tcount[lev], kGemmThreads, S.smem_gemm, s>>>(
        S.E, S.shift_tiles.as<ShiftTile>() + S.l2l_tfirst[lev], S.shift_cols.as<ShiftCol>(), S.shift_ops->as<T>(),
        reinterpret_cast<const T*>(Lx), reinterpret_cast<T*>(Lx));
    BP_LAUNCH_CHECK();
    end(1);
  }
  for (int lev = 0; lev < nlev; ++lev) join_x(lev);  // every level stream rejoins the FMM stream
  begin(5, s);
  {
    const int NT = S.nt, EQ = (NT + 3) * (NT + 4) / 2;
    prep_csr_kernel<T><<<S.n_leaf, 256, S.smem_csr, s>>>(S.E, EQ, S.leaf_items.as<LeafItem>(), S.prep_rowptr->as<int>(),
                                                          S.prep_cols->as<int>(), S.prep_vals->as<T>(),
                                                          reinterpret_cast<const T*>(Lx),
                                                          reinterpret_cast<T*>(S.leaf_exp.as<C>()));
    BP_LAUNCH_CHECK();
  }
  end(1);
  begin(7, s);
  launch_k(pdl_ok, l2p_eval_kernel<T>, S.n_eval, kEvalThreads, S.smem_eval, s, S.nt,
           (const LeafItem*)S.eval_items.as<LeafItem>(), contents, (const double*)P.d_normal.as<double>(),
           (const C*)S.leaf_exp.as<C>(), (const C*)S.eval_basis.as<C>(), P.n, y);
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
