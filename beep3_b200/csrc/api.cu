// C ABI entry points (declared in include/beep3_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <future>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"

namespace bp {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

namespace {

Ctx* as_ctx(bp_ctx c) { return reinterpret_cast<Ctx*>(c); }
Problem* as_problem(bp_problem p) { return reinterpret_cast<Problem*>(p); }

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) BP_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// [n][7] points (x y z nx ny nz w) -> 7 arrays of n values, FP32 copy too
// when soa_f is set; *bad is set when a value is not finite.
__global__ void aos_to_soa_kernel(const double* __restrict__ aos, int n, double* __restrict__ soa,
                                  float* __restrict__ soa_f, int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool ok = true;
  for (int f = 0; f < 7; ++f) {
    const double v = aos[7 * (size_t)i + f];
    ok = ok && isfinite(v);
    soa[(size_t)f * n + i] = v;
    if (soa_f) soa_f[(size_t)f * n + i] = (float)v;
  }
  if (!ok) atomicOr(bad, 1);
}

// A patch point list: offsets checked on the host, the points uploaded as
// given and laid out (and checked) on the device.
void upload_points(Ctx* c, const char* what, int n, const int32_t* off, const double* pts,
                   std::vector<int32_t>& h_off, int& n_pts, DevBuf& soa, DevBuf* soa_f) {
  if (!off || !pts) throw std::invalid_argument(std::string(what) + ": missing point list");
  h_off.assign(off, off + n + 1);
  if (h_off[0] != 0) throw std::invalid_argument(std::string(what) + ": offsets must start at 0");
  for (int i = 0; i < n; ++i)
    if (h_off[i + 1] <= h_off[i]) throw std::invalid_argument(std::string(what) + ": every patch needs points");
  n_pts = h_off[n];
  DevBuf aos(c, sizeof(double) * 7 * (size_t)n_pts);
  DevBuf bad(c, sizeof(int));
  BP_CUDA(cudaMemcpyAsync(aos.get(), pts, aos.bytes(), cudaMemcpyHostToDevice, c->stream));
  BP_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), c->stream));
  soa.alloc(c, sizeof(double) * 7 * (size_t)n_pts);
  if (soa_f) soa_f->alloc(c, sizeof(float) * 7 * (size_t)n_pts);
  aos_to_soa_kernel<<<(n_pts + 255) / 256, 256, 0, c->stream>>>(aos.as<double>(), n_pts, soa.as<double>(),
                                                                 soa_f ? soa_f->as<float>() : nullptr, bad.as<int>());
  BP_LAUNCH_CHECK();
  int h_bad = 0;
  BP_CUDA(cudaMemcpyAsync(&h_bad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BP_CUDA(cudaStreamSynchronize(c->stream));
  if (h_bad) throw std::invalid_argument(std::string(what) + ": non-finite point data");
}

int32_t check_params(const char* who, const bp_params* prm) {
  if (prm->precision != BP_PREC_FP64 && prm->precision != BP_PREC_MIXED)
    return fail(BP_ERR_INVALID, std::string(who) + ": unknown precision");
  if (!(prm->kappa >= 0.0) || !std::isfinite(prm->kappa)) return fail(BP_ERR_INVALID, std::string(who) + ": bad kappa");
  if (prm->flags &
      ~(BP_FLAG_NEARFIELD_ON_DEMAND | BP_FLAG_DEVICE_TREE | BP_FLAG_COMPACT_NEARFIELD | BP_FLAG_MESH_PAIR_CACHE))
    return fail(BP_ERR_INVALID, std::string(who) + ": unknown flags");
  if ((prm->flags & BP_FLAG_COMPACT_NEARFIELD) &&
      (prm->precision != BP_PREC_MIXED || (prm->flags & BP_FLAG_NEARFIELD_ON_DEMAND)))
    return fail(BP_ERR_INVALID,
                std::string(who) + ": the compact near field needs the mixed engine and cached coefficients");
  if (prm->nbsize <= 0) return fail(BP_ERR_INVALID, std::string(who) + ": nbsize must be positive");
  if (prm->nterms != 9)
    return fail(BP_ERR_UNSUPPORTED, std::string(who) +
                                        ": FMM order must be 9 (the reference's BEM matvec order; the far-field "
                                        "kernels' thread and shared-memory layouts are sized for it)");
  return BP_OK;
}

// One tree of the scenarios' trees: level by level, scenario after
// scenario, node links and contents renumbered (scenario s's patch i is the
// problem's patch first[s] + i).  Neighbours never cross scenarios, so the
// near field and the FMM's interaction lists stay inside each scenario; the
// per-level operators are shared because every scenario's cube has the same
// edge.
void merge_forest(const std::vector<TreeInfo>& F, const std::vector<int>& first, TreeInfo& out) {
  const int S = (int)F.size();
  out = TreeInfo();
  for (const TreeInfo& t : F) out.n_levels = std::max(out.n_levels, t.n_levels);
  std::vector<std::vector<int>> remap(S);
  for (int s = 0; s < S; ++s) remap[s].assign(F[s].nodes.size(), -1);
  out.level_start.assign(out.n_levels + 1, 0);
  for (int l = 0; l < out.n_levels; ++l) {
    out.level_start[l] = (int)out.nodes.size();
    for (int s = 0; s < S; ++s) {
      if (l >= F[s].n_levels) continue;
      for (int j = F[s].level_start[l]; j < F[s].level_start[l + 1]; ++j) {
        remap[s][j] = (int)out.nodes.size();
        out.nodes.push_back(F[s].nodes[j]);
      }
    }
  }
  out.level_start[out.n_levels] = (int)out.nodes.size();
  out.n_mp_per_level.assign(out.n_levels, 0);
  out.n_lc_per_level.assign(out.n_levels, 0);
  for (int s = 0; s < S; ++s) {
    const TreeInfo& t = F[s];
    for (size_t j = 0; j < t.nodes.size(); ++j) {
      TreeNode& nd = out.nodes[remap[s][j]];
      auto re = [&](int32_t k) { return k < 0 ? -1 : remap[s][k]; };
      nd.parent = re(nd.parent);
      for (int c = 0; c < 8; ++c) nd.children[c] = re(nd.children[c]);
      for (int nb = 0; nb < 27; ++nb) nd.neighbours[nb] = re(nd.neighbours[nb]);
    }
  }
  // contents, node by node in the merged order; FMM slots per merged level
  for (int l = out.n_levels - 1; l >= 0; --l)
    for (int j = out.level_start[l]; j < out.level_start[l + 1]; ++j) {
      TreeNode& nd = out.nodes[j];
      nd.lc_idx = (nd.flags & TREE_SHADOW) ? -1 : out.n_lc_per_level[l]++;
      nd.mp_idx = nd.content_count > 0 ? out.n_mp_per_level[l]++ : -1;
    }
  std::vector<int> owner(out.nodes.size(), 0);
  for (int s = 0; s < S; ++s)
    for (int k : remap[s]) owner[k] = s;
  for (size_t j = 0; j < out.nodes.size(); ++j) {
    TreeNode& nd = out.nodes[j];
    const int s = owner[j];
    const int64_t src = nd.content_start;
    nd.content_start = (int64_t)out.contents.size();
    for (int32_t q = 0; q < nd.content_count; ++q) out.contents.push_back(first[s] + F[s].contents[src + q]);
  }
}

// The steps after the patch geometry is in place (host arrays and device
// point lists): tree, per-patch device arrays, near field, FMM, matvec graph.
void finish_problem(Ctx* c, Problem& P) {
  auto t0 = std::chrono::steady_clock::now();
  P.d_centroid = upload(c, P.h_centroid);
  if (P.scen_first.empty()) {
    P.scen_first = {0, P.n};
    P.scen_centre.assign(P.params.cube_centre, P.params.cube_centre + 3);
  }
  const int S = P.n_scen();
  std::vector<TreeInfo> forest(S);
  auto one_tree = [&](int s) {
    const int a = P.scen_first[s], n = P.scen_first[s + 1] - a;
    if (P.params.flags & BP_FLAG_DEVICE_TREE)
      build_device_tree(c, P.d_centroid.as<double>() + 3 * (size_t)a, n, &P.scen_centre[3 * s], P.params.cube_edge,
                        P.params.nbsize, S == 1 ? P.tree : forest[s]);
    else
      build_reference_tree(P.h_centroid.data() + 3 * (size_t)a, n, &P.scen_centre[3 * s], P.params.cube_edge,
                           P.params.nbsize, S == 1 ? P.tree : forest[s]);
  };
  if (S == 1) {
    one_tree(0);
  } else {
    if (P.params.flags & BP_FLAG_DEVICE_TREE) {
      for (int s = 0; s < S; ++s) one_tree(s);
    } else {  // host trees of the scenarios side by side
      std::vector<std::future<void>> jobs;
      for (int s = 0; s < S; ++s) jobs.push_back(std::async(std::launch::async, one_tree, s));
      for (auto& j : jobs) j.get();
    }
    merge_forest(forest, P.scen_first, P.tree);
  }
  P.tree_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  P.d_normal = upload(c, P.h_normal);
  P.d_area = upload(c, P.h_area);
  P.d_eps = upload(c, P.h_eps);
  P.d_qual_off = upload(c, P.h_qual_off);
  P.d_quad_off = upload(c, P.h_quad_off);
  P.d_gal_off = upload(c, P.h_gal_off);
  P.d_x.alloc(c, sizeof(double) * 2 * (size_t)P.n);
  P.d_y.alloc(c, sizeof(double) * 2 * (size_t)P.n);
  nf_build_structure(P);
  nf_assemble(P);
  auto t1 = std::chrono::steady_clock::now();
  if (fmm_active(P)) fmm_setup(P);  // host work overlaps the assembly kernels
  P.fmm_setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
  nf_join(P);
  matvec_setup(P);
  BP_CUDA(cudaStreamSynchronize(c->stream));
  P.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  float ms = 0.f;
  BP_CUDA(cudaEventElapsedTime(&ms, P.asm_t0, P.asm_t1));
  P.assemble_ms = ms;
}

// p -> R (p - c) + o and n -> R n of `count` points of a 7-array SoA list
// (x y z nx ny nz w, row stride src_n) into rows [base, base + count) of a
// list of row stride dst_n; FP32 copy too when dst_f is set.
struct Rigid {
  double R[9], c[3], o[3];
};
__global__ void place_points_kernel(const double* __restrict__ src, int src_n, double* __restrict__ dst, int dst_n,
                                    int base, int count, Rigid rg, float* __restrict__ dst_f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double x = src[i] - rg.c[0], y = src[src_n + i] - rg.c[1], z = src[2 * (size_t)src_n + i] - rg.c[2];
  const double nx = src[3 * (size_t)src_n + i], ny = src[4 * (size_t)src_n + i], nz = src[5 * (size_t)src_n + i];
  double v[7];
  for (int r = 0; r < 3; ++r) {
    v[r] = rg.R[3 * r] * x + rg.R[3 * r + 1] * y + rg.R[3 * r + 2] * z + rg.o[r];
    v[3 + r] = rg.R[3 * r] * nx + rg.R[3 * r + 1] * ny + rg.R[3 * r + 2] * nz;
  }
  v[6] = src[6 * (size_t)src_n + i];
  for (int f = 0; f < 7; ++f) {
    dst[(size_t)f * dst_n + base + i] = v[f];
    if (dst_f) dst_f[(size_t)f * dst_n + base + i] = (float)v[f];
  }
}

}  // namespace
}  // namespace bp

using namespace bp;

extern "C" {

BP_API const char* bp_last_error(void) { return g_last_error.c_str(); }
BP_API int32_t bp_abi_version(void) { return BP_ABI_VERSION; }

BP_API int32_t bp_ctx_create(int32_t device, uint64_t hbm_budget_bytes, bp_ctx* out) {
  return guarded_engine([&]() -> int32_t {
    if (!out) return fail(BP_ERR_INVALID, "bp_ctx_create: null out");
    int ndev = 0;
    BP_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(BP_ERR_INVALID, "bp_ctx_create: no such device");
    DeviceGuard g(device);
    auto c = new Ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    BP_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    BP_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    *out = reinterpret_cast<bp_ctx>(c);
    return BP_OK;
  });
}

BP_API int32_t bp_ctx_destroy(bp_ctx ctx) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = as_ctx(ctx);
    if (!c) return BP_OK;
    if (c->live_problems.load() > 0 || c->live_meshes.load() > 0)
      return fail(BP_ERR_INVALID, "bp_ctx_destroy: " + std::to_string(c->live_problems.load()) + " problem(s) and " +
                                      std::to_string(c->live_meshes.load()) +
                                      " mesh(es) of this context are still alive; destroy them first");
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    c->fmm_plans.clear();  // their device blocks go back to the cache
    c->trim();             // the released blocks kept for reuse
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return BP_OK;
  });
}

BP_API int32_t bp_ctx_set_stream(bp_ctx ctx, void* stream) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = as_ctx(ctx);
    if (!c) return fail(BP_ERR_INVALID, "bp_ctx_set_stream: null context");
    cudaStream_t next = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    if (next == c->stream) return BP_OK;
    // device blocks released by work still pending on the old stream go back
    // to the context's cache; work on the new stream may take them, so the
    // old stream's work must be finished first
    DeviceGuard g(c->device);
    BP_CUDA(cudaStreamSynchronize(c->stream));
    c->stream = next;
    return BP_OK;
  });
}

BP_API int32_t bp_ctx_memory(bp_ctx ctx, uint64_t* used, uint64_t* budget) {
  Ctx* c = as_ctx(ctx);
  if (!c) return fail(BP_ERR_INVALID, "bp_ctx_memory: null context");
  if (used) *used = c->used;
  if (budget) *budget = c->budget;
  return BP_OK;
}

BP_API int32_t bp_ctx_cache(bp_ctx ctx, uint64_t* cached, int32_t release) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = as_ctx(ctx);
    if (!c) return fail(BP_ERR_INVALID, "bp_ctx_cache: null context");
    if (release) {
      DeviceGuard g(c->device);
      BP_CUDA(cudaStreamSynchronize(c->stream));
      c->trim();
    }
    if (cached) {
      std::lock_guard<std::mutex> lk(c->mu);
      *cached = c->cached;
    }
    return BP_OK;
  });
}

BP_API int32_t bp_ctx_synchronize(bp_ctx ctx) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = as_ctx(ctx);
    if (!c) return fail(BP_ERR_INVALID, "bp_ctx_synchronize: null context");
    DeviceGuard g(c->device);
    BP_CUDA(cudaStreamSynchronize(c->stream));
    return BP_OK;
  });
}

BP_API int32_t bp_problem_create(bp_ctx ctx, const bp_patches* pp, const bp_params* prm, bp_problem* out) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = as_ctx(ctx);
    if (!c || !pp || !prm || !out) return fail(BP_ERR_INVALID, "bp_problem_create: null argument");
    const int n = pp->n_patches;
    if (n <= 0) return fail(BP_ERR_INVALID, "bp_problem_create: no patches");
    if (!pp->centroid || !pp->normal || !pp->area || !pp->dielectric_ratio)
      return fail(BP_ERR_INVALID, "bp_problem_create: missing patch arrays");
    if (const int32_t e = check_params("bp_problem_create", prm)) return e;
    DeviceGuard g(c->device);
    auto P = std::make_unique<Problem>();
    P->ctx = c;
    P->live.attach(c->live_problems);
    P->n = n;
    P->params = *prm;
    P->fp64 = prm->precision == BP_PREC_FP64;
    P->h_centroid.assign(pp->centroid, pp->centroid + 3 * (size_t)n);
    P->h_normal.assign(pp->normal, pp->normal + 3 * (size_t)n);
    P->h_area.assign(pp->area, pp->area + n);
    P->h_eps.assign(pp->dielectric_ratio, pp->dielectric_ratio + n);
    P->h_gc.assign(n, 0.5);
    if (pp->gc) P->h_gc.assign(pp->gc, pp->gc + n);
    for (int i = 0; i < n; ++i) {
      if (!(P->h_eps[i] > 0)) return fail(BP_ERR_INVALID, "bp_problem_create: dielectric ratio must be > 0");
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(P->h_centroid[3 * i + k]) || !std::isfinite(P->h_normal[3 * i + k]))
          return fail(BP_ERR_INVALID, "bp_problem_create: non-finite patch geometry");
    }
    upload_points(c, "qualocation", n, pp->qual_offsets, pp->qual_points, P->h_qual_off, P->n_qual_pts, P->d_qual,
                  P->fp64 ? nullptr : &P->d_qual_f);
    upload_points(c, "quadrature", n, pp->quad_offsets, pp->quad_points, P->h_quad_off, P->n_quad_pts, P->d_quad,
                  P->fp64 ? nullptr : &P->d_quad_f);
    upload_points(c, "galerkin", n, pp->galerkin_offsets, pp->galerkin_points, P->h_gal_off, P->n_gal_pts, P->d_gal,
                  nullptr);
    finish_problem(c, *P);
    *out = reinterpret_cast<bp_problem>(P.release());
    return BP_OK;
  });
}

BP_API int32_t bp_mesh_create(bp_ctx ctx, const bp_patches* pp, const double centre[3], bp_mesh* out) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = as_ctx(ctx);
    if (!c || !pp || !centre || !out) return fail(BP_ERR_INVALID, "bp_mesh_create: null argument");
    const int n = pp->n_patches;
    if (n <= 0) return fail(BP_ERR_INVALID, "bp_mesh_create: no patches");
    if (!pp->centroid || !pp->normal || !pp->area) return fail(BP_ERR_INVALID, "bp_mesh_create: missing patch arrays");
    DeviceGuard g(c->device);
    auto m = std::make_unique<DevMesh>();
    m->ctx = c;
    m->live.attach(c->live_meshes);
    m->n = n;
    for (int k = 0; k < 3; ++k) {
      if (!std::isfinite(centre[k])) return fail(BP_ERR_INVALID, "bp_mesh_create: non-finite centre");
      m->centre[k] = centre[k];
    }
    m->h_centroid.assign(pp->centroid, pp->centroid + 3 * (size_t)n);
    m->h_normal.assign(pp->normal, pp->normal + 3 * (size_t)n);
    m->h_area.assign(pp->area, pp->area + n);
    m->h_gc.assign(n, 0.5);
    if (pp->gc) m->h_gc.assign(pp->gc, pp->gc + n);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(m->h_centroid[3 * i + k]) || !std::isfinite(m->h_normal[3 * i + k]))
          return fail(BP_ERR_INVALID, "bp_mesh_create: non-finite patch geometry");
    upload_points(c, "qualocation", n, pp->qual_offsets, pp->qual_points, m->h_qual_off, m->n_qual_pts, m->d_qual,
                  nullptr);
    upload_points(c, "quadrature", n, pp->quad_offsets, pp->quad_points, m->h_quad_off, m->n_quad_pts, m->d_quad,
                  nullptr);
    upload_points(c, "galerkin", n, pp->galerkin_offsets, pp->galerkin_points, m->h_gal_off, m->n_gal_pts, m->d_gal,
                  nullptr);
    *out = reinterpret_cast<bp_mesh>(m.release());
    return BP_OK;
  });
}

BP_API int32_t bp_mesh_destroy(bp_mesh mesh) {
  return guarded_engine([&]() -> int32_t {
    DevMesh* m = reinterpret_cast<DevMesh*>(mesh);
    if (!m) return BP_OK;
    {
      std::lock_guard<std::mutex> lk(m->mu);
      if (m->users > 0) {  // the last posed problem placed from it deletes it
        m->destroy_pending = true;
        return BP_OK;
      }
    }
    DeviceGuard g(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    delete m;
    return BP_OK;
  });
}

// A problem from placed mesh instances; scen_inst (n_scen + 1 instance
// offsets, null for one scenario) and centres (3 n_scen) split it into
// independent scenarios.
static int32_t create_posed(Ctx* c, const bp_instance* inst, int32_t n_inst, const bp_params* prm,
                            const int32_t* scen_inst, int32_t n_scen, const double* centres, bp_problem* out) {
  {
    if (!c || !inst || !prm || !out || n_inst <= 0) return fail(BP_ERR_INVALID, "bp_problem_create_posed: bad argument");
    if (const int32_t e = check_params("bp_problem_create_posed", prm)) return e;
    long long n_total = 0, nq = 0, nd = 0, ng = 0;
    for (int q = 0; q < n_inst; ++q) {
      const DevMesh* m = reinterpret_cast<const DevMesh*>(inst[q].mesh);
      if (!m || m->ctx != c) return fail(BP_ERR_INVALID, "bp_problem_create_posed: mesh of another context");
      if (!(inst[q].dielectric_ratio > 0) || !std::isfinite(inst[q].dielectric_ratio))
        return fail(BP_ERR_INVALID, "bp_problem_create_posed: dielectric ratio must be > 0");
      for (int k = 0; k < 9; ++k)
        if (!std::isfinite(inst[q].rotation[k])) return fail(BP_ERR_INVALID, "bp_problem_create_posed: bad rotation");
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(inst[q].offset[k])) return fail(BP_ERR_INVALID, "bp_problem_create_posed: bad offset");
      n_total += m->n;
      nq += m->n_qual_pts;
      nd += m->n_quad_pts;
      ng += m->n_gal_pts;
    }
    if (n_total > (1LL << 30) || nq > (1LL << 31) - 1 || nd > (1LL << 31) - 1 || ng > (1LL << 31) - 1)
      return fail(BP_ERR_INVALID, "bp_problem_create_posed: too many patches or points");
    DeviceGuard g(c->device);
    auto P = std::make_unique<Problem>();
    P->ctx = c;
    P->live.attach(c->live_problems);
    P->n = (int)n_total;
    P->params = *prm;
    P->fp64 = prm->precision == BP_PREC_FP64;
    P->n_qual_pts = (int)nq;
    P->n_quad_pts = (int)nd;
    P->n_gal_pts = (int)ng;
    P->d_qual.alloc(c, sizeof(double) * 7 * (size_t)nq);
    P->d_quad.alloc(c, sizeof(double) * 7 * (size_t)nd);
    P->d_gal.alloc(c, sizeof(double) * 7 * (size_t)ng);
    if (!P->fp64) {
      P->d_qual_f.alloc(c, sizeof(float) * 7 * (size_t)nq);
      P->d_quad_f.alloc(c, sizeof(float) * 7 * (size_t)nd);
    }
    P->h_qual_off.assign(1, 0);
    P->h_quad_off.assign(1, 0);
    P->h_gal_off.assign(1, 0);
    int bq = 0, bd = 0, bg = 0;
    for (int q = 0; q < n_inst; ++q) {
      const DevMesh& m = *reinterpret_cast<const DevMesh*>(inst[q].mesh);
      Rigid rg;
      for (int k = 0; k < 9; ++k) rg.R[k] = inst[q].rotation[k];
      for (int k = 0; k < 3; ++k) {
        rg.c[k] = m.centre[k];
        rg.o[k] = inst[q].offset[k];
      }
      Placement pl;
      pl.mesh = reinterpret_cast<DevMesh*>(inst[q].mesh);
      for (int k = 0; k < 9; ++k) pl.R[k] = rg.R[k];
      for (int k = 0; k < 3; ++k) {
        pl.c[k] = rg.c[k];
        pl.o[k] = rg.o[k];
      }
      pl.q_begin = bq;
      pl.q_count = m.n_qual_pts;
      P->placements.push_back(pl);
      mesh_acquire(pl.mesh);
      // patch centres and normals on the host (the tree is built there)
      for (int i = 0; i < m.n; ++i) {
        const double* p = &m.h_centroid[3 * (size_t)i];
        const double* nv = &m.h_normal[3 * (size_t)i];
        const double x = p[0] - rg.c[0], y = p[1] - rg.c[1], z = p[2] - rg.c[2];
        for (int r = 0; r < 3; ++r) {
          P->h_centroid.push_back(rg.R[3 * r] * x + rg.R[3 * r + 1] * y + rg.R[3 * r + 2] * z + rg.o[r]);
          P->h_normal.push_back(rg.R[3 * r] * nv[0] + rg.R[3 * r + 1] * nv[1] + rg.R[3 * r + 2] * nv[2]);
        }
      }
      P->h_area.insert(P->h_area.end(), m.h_area.begin(), m.h_area.end());
      P->h_gc.insert(P->h_gc.end(), m.h_gc.begin(), m.h_gc.end());
      P->h_eps.insert(P->h_eps.end(), (size_t)m.n, inst[q].dielectric_ratio);
      for (int i = 1; i <= m.n; ++i) {
        P->h_qual_off.push_back(bq + m.h_qual_off[i]);
        P->h_quad_off.push_back(bd + m.h_quad_off[i]);
        P->h_gal_off.push_back(bg + m.h_gal_off[i]);
      }
      // point lists: placed on the device
      auto place = [&](const DevBuf& src, int src_n, DevBuf& dst, int dst_n, int base, float* dst_f) {
        if (src_n == 0) return;
        place_points_kernel<<<(src_n + 255) / 256, 256, 0, c->stream>>>(src.as<double>(), src_n, dst.as<double>(),
                                                                       dst_n, base, src_n, rg, dst_f);
        BP_LAUNCH_CHECK();
      };
      place(m.d_qual, m.n_qual_pts, P->d_qual, (int)nq, bq, P->fp64 ? nullptr : P->d_qual_f.as<float>());
      place(m.d_quad, m.n_quad_pts, P->d_quad, (int)nd, bd, P->fp64 ? nullptr : P->d_quad_f.as<float>());
      place(m.d_gal, m.n_gal_pts, P->d_gal, (int)ng, bg, nullptr);
      bq += m.n_qual_pts;
      bd += m.n_quad_pts;
      bg += m.n_gal_pts;
    }
    if (scen_inst) {
      P->scen_first.assign(1, 0);
      int q = 0;
      for (int s = 0; s < n_scen; ++s) {
        int n_s = 0;
        for (; q < scen_inst[s + 1]; ++q) {
          P->placements[q].scenario = s;
          n_s += reinterpret_cast<const DevMesh*>(inst[q].mesh)->n;
        }
        P->scen_first.push_back(P->scen_first.back() + n_s);
      }
      P->scen_centre.assign(centres, centres + 3 * (size_t)n_scen);
    }
    finish_problem(c, *P);
    *out = reinterpret_cast<bp_problem>(P.release());
    return BP_OK;
  }
}

BP_API int32_t bp_problem_create_posed(bp_ctx ctx, const bp_instance* inst, int32_t n_inst, const bp_params* prm,
                                       bp_problem* out) {
  return guarded_engine([&]() -> int32_t { return create_posed(as_ctx(ctx), inst, n_inst, prm, nullptr, 1, nullptr, out); });
}

BP_API int32_t bp_problem_create_batch(bp_ctx ctx, const bp_instance* inst, int32_t n_inst,
                                       const int32_t* scenario_first, int32_t n_scenarios, const double* cube_centres,
                                       const bp_params* prm, bp_problem* out) {
  return guarded_engine([&]() -> int32_t {
    if (!scenario_first || !cube_centres || n_scenarios <= 0 || !prm)
      return fail(BP_ERR_INVALID, "bp_problem_create_batch: bad argument");
    if (scenario_first[0] != 0 || scenario_first[n_scenarios] != n_inst)
      return fail(BP_ERR_INVALID, "bp_problem_create_batch: scenario_first must run from 0 to n_inst");
    for (int s = 0; s < n_scenarios; ++s)
      if (scenario_first[s + 1] <= scenario_first[s])
        return fail(BP_ERR_INVALID, "bp_problem_create_batch: every scenario needs an instance");
    for (int k = 0; k < 3 * n_scenarios; ++k)
      if (!std::isfinite(cube_centres[k])) return fail(BP_ERR_INVALID, "bp_problem_create_batch: non-finite centre");
    return create_posed(as_ctx(ctx), inst, n_inst, prm, scenario_first, n_scenarios, cube_centres, out);
  });
}

BP_API int32_t bp_problem_destroy(bp_problem p) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P) return BP_OK;
    DeviceGuard g(P->ctx->device);
    cudaStreamSynchronize(P->ctx->stream);
    delete P;
    return BP_OK;
  });
}

BP_API int32_t bp_problem_info_get(bp_problem p, bp_problem_info* info) {
  Problem* P = as_problem(p);
  if (!P || !info) return fail(BP_ERR_INVALID, "bp_problem_info_get: null argument");
  info->n_patches = P->n;
  info->n_levels = P->tree.n_levels;
  info->n_nodes = (int64_t)P->tree.nodes.size();
  info->n_leaves = P->nf.n_leaves;
  info->n_nearfield_pairs = P->nf.n_pairs;
  info->n_nearfield_cols = P->nf.h_col_off.empty() ? 0 : P->nf.h_col_off.back();
  info->fmm_active = fmm_active(*P) ? 1 : 0;
  info->device_bytes = P->ctx->used;
  info->tree_ms = P->tree_ms;
  info->assemble_ms = P->assemble_ms;
  info->fmm_setup_ms = P->fmm_setup_ms;
  info->setup_ms = P->setup_ms;
  info->gmres_graph = P->gmres_graph ? 1 : 0;
  info->n_scenarios = P->n_scen();
  const FmmWork w = fmm_work(*P);
  info->fmm_m2x_cols = w.m2x_cols;
  info->fmm_x2l_cols = w.x2l_cols;
  info->fmm_translations = w.xl_entries;
  info->fmm_shift_cols = w.shift_cols;
  info->fmm_plane_waves = w.plane_waves;
  info->fmm_coefficients = w.coefficients;
  return BP_OK;
}

static int32_t export_tree(const TreeInfo& T, int32_t* n_nodes, int32_t* n_levels, int64_t* n_contents, int32_t* node_info,
                           double* node_geom, int32_t* contents) {
  if (n_nodes) *n_nodes = (int32_t)T.nodes.size();
  if (n_contents) *n_contents = (int64_t)T.contents.size();
  if (n_levels) *n_levels = T.n_levels;
  for (size_t k = 0; k < T.nodes.size(); ++k) {
    const TreeNode& nd = T.nodes[k];
    if (node_info) {
      int32_t* o = node_info + 18 * k;
      o[0] = nd.level;
      o[1] = (int32_t)nd.ix;
      o[2] = (int32_t)nd.iy;
      o[3] = (int32_t)nd.iz;
      o[4] = nd.flags;
      o[5] = nd.parent;
      o[6] = (int32_t)nd.content_start;
      o[7] = nd.content_count;
      o[8] = nd.mp_idx;
      o[9] = nd.lc_idx;
      for (int c = 0; c < 8; ++c) o[10 + c] = nd.children[c];
    }
    if (node_geom) {
      for (int d = 0; d < 3; ++d) node_geom[4 * k + d] = nd.centre[d];
      node_geom[4 * k + 3] = nd.edge;
    }
  }
  if (contents) std::copy(T.contents.begin(), T.contents.end(), contents);
  return BP_OK;
}

BP_API int32_t bp_problem_tree(bp_problem p, int32_t* n_nodes, int32_t* n_levels, int64_t* n_contents, int32_t* node_info,
                               double* node_geom, int32_t* contents) {
  Problem* P = as_problem(p);
  if (!P) return fail(BP_ERR_INVALID, "bp_problem_tree: null problem");
  return export_tree(P->tree, n_nodes, n_levels, n_contents, node_info, node_geom, contents);
}

BP_API int32_t bp_tree_create(int32_t n, const double* points, const double cube_centre[3], double cube_edge,
                              int32_t nbsize, bp_tree* out) {
  return guarded([&]() -> int32_t {
    if (n <= 0 || !points || !cube_centre || !out) return fail(BP_ERR_INVALID, "bp_tree_create: bad argument");
    auto T = std::make_unique<TreeInfo>();
    build_reference_tree(points, n, cube_centre, cube_edge, nbsize, *T);
    *out = reinterpret_cast<bp_tree>(T.release());
    return BP_OK;
  });
}

BP_API int32_t bp_tree_export(bp_tree t, int32_t* n_nodes, int32_t* n_levels, int64_t* n_contents, int32_t* node_info, double* node_geom,
                              int32_t* contents) {
  if (!t) return fail(BP_ERR_INVALID, "bp_tree_export: null tree");
  return export_tree(*reinterpret_cast<TreeInfo*>(t), n_nodes, n_levels, n_contents, node_info, node_geom, contents);
}

BP_API int32_t bp_tree_destroy(bp_tree t) {
  delete reinterpret_cast<TreeInfo*>(t);
  return BP_OK;
}

BP_API int32_t bp_matvec_device(bp_problem p, const double* x_dev, double* y_dev) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !x_dev || !y_dev) return fail(BP_ERR_INVALID, "bp_matvec_device: null argument");
    if (x_dev == y_dev) return fail(BP_ERR_INVALID, "bp_matvec_device: x and y must not alias");
    DeviceGuard g(P->ctx->device);
    matvec_device(*P, x_dev, y_dev);
    return BP_OK;
  });
}

BP_API int32_t bp_matvec_profile(bp_problem p, const double* x_dev, double* y_dev, int32_t reps, double* stage_ms,
                                 int32_t* stage_launches, int32_t* n_stages) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !x_dev || !y_dev || !stage_ms || reps <= 0) return fail(BP_ERR_INVALID, "bp_matvec_profile: bad argument");
    DeviceGuard g(P->ctx->device);
    StageTimes st;
    for (int r = 0; r < reps; ++r) matvec_device(*P, x_dev, y_dev, &st);
    BP_CUDA(cudaStreamSynchronize(P->ctx->stream));
    for (int s = 0; s < kStages; ++s) {
      stage_ms[s] = st.ms(s) / reps;
      if (stage_launches) stage_launches[s] = st.launches[s] / reps;
    }
    if (n_stages) *n_stages = kStages;
    return BP_OK;
  });
}

BP_API int32_t bp_matvec(bp_problem p, const double* x, double* y) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !x || !y) return fail(BP_ERR_INVALID, "bp_matvec: null argument");
    DeviceGuard g(P->ctx->device);
    const size_t bytes = sizeof(double) * 2 * (size_t)P->n;
    cudaStream_t st = P->ctx->stream;
    // straight into and out of the matvec graph's own buffers, and the
    // far field's timeout word read back behind y: one synchronisation
    BP_CUDA(cudaMemcpyAsync(P->d_gx.get(), x, bytes, cudaMemcpyHostToDevice, st));
    matvec_device(*P, P->d_gx.as<double>(), P->d_gy.as<double>());
    BP_CUDA(cudaMemcpyAsync(y, P->d_gy.get(), bytes, cudaMemcpyDeviceToHost, st));
    const int* sd = fmm_status_dev(*P);
    if (sd) BP_CUDA(cudaMemcpyAsync(P->h_status, sd, sizeof(int), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    fmm_raise_if(*P, sd ? *P->h_status : 0);
    return BP_OK;
  });
}

BP_API int32_t bp_solve_device(bp_problem p, const double* rhs_dev, double* x_dev, double tol, int32_t max_iters,
                               int32_t restart, int32_t* iterations, double* rel_residual) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !rhs_dev || !x_dev) return fail(BP_ERR_INVALID, "bp_solve_device: null argument");
    if (!(tol > 0)) return fail(BP_ERR_INVALID, "bp_solve_device: tol must be positive");
    DeviceGuard g(P->ctx->device);
    std::vector<double> rr(P->n_scen(), 0.0);
    const bool x0 = device_all_zero(*P, x_dev, 2 * (int64_t)P->n);
    int its = gmres_device(*P, rhs_dev, x_dev, tol, max_iters, restart, rr.data(), nullptr, x0);
    const double worst = *std::max_element(rr.begin(), rr.end());
    if (iterations) *iterations = its;
    if (rel_residual) *rel_residual = worst;
    if (worst > tol) return fail(BP_ERR_NOT_CONVERGED, "GMRES reached its iteration limit");
    return BP_OK;
  });
}

// bp_solve (worst scenario's iterations and residual) and bp_solve_batch
// (one entry per scenario in iterations and rel_residual)
static int32_t solve_host(bp_problem p, const double* rhs, double* x, double tol, int32_t max_iters, int32_t restart,
                          int32_t* iterations, double* rel_residual, bool scenario_out) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !rhs || !x) return fail(BP_ERR_INVALID, "bp_solve: null argument");
    if (!(tol > 0)) return fail(BP_ERR_INVALID, "bp_solve: tol must be positive");
    DeviceGuard g(P->ctx->device);
    const size_t bytes = sizeof(double) * 2 * (size_t)P->n;
    cudaStream_t st = P->ctx->stream;
    DevBuf& b = P->scratch_b;
    if (b.bytes() < bytes) b.alloc(P->ctx, bytes);
    BP_CUDA(cudaMemcpyAsync(b.get(), rhs, bytes, cudaMemcpyHostToDevice, st));
    const bool x0 = std::all_of(x, x + 2 * (size_t)P->n, [](double v) { return v == 0.0; });
    if (x0)  // a zero initial guess (the usual one) is set on the device, not copied
      BP_CUDA(cudaMemsetAsync(P->d_x.get(), 0, bytes, st));
    else
      BP_CUDA(cudaMemcpyAsync(P->d_x.get(), x, bytes, cudaMemcpyHostToDevice, st));
    std::vector<double> rr(P->n_scen(), 0.0);
    std::vector<int> its(P->n_scen(), 0);
    gmres_device(*P, b.as<double>(), P->d_x.as<double>(), tol, max_iters, restart, rr.data(), its.data(), x0);
    BP_CUDA(cudaMemcpyAsync(x, P->d_x.get(), bytes, cudaMemcpyDeviceToHost, st));
    const int* sd = fmm_status_dev(*P);
    if (sd) BP_CUDA(cudaMemcpyAsync(P->h_status, sd, sizeof(int), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    fmm_raise_if(*P, sd ? *P->h_status : 0);
    const double worst = *std::max_element(rr.begin(), rr.end());
    if (scenario_out) {  // bp_solve_batch: per scenario
      std::copy(its.begin(), its.end(), iterations);
      std::copy(rr.begin(), rr.end(), rel_residual);
    } else {
      if (iterations) *iterations = *std::max_element(its.begin(), its.end());
      if (rel_residual) *rel_residual = worst;
    }
    if (worst > tol) return fail(BP_ERR_NOT_CONVERGED, "GMRES reached its iteration limit");
    return BP_OK;
  });
}

BP_API int32_t bp_solve(bp_problem p, const double* rhs, double* x, double tol, int32_t max_iters, int32_t restart,
                        int32_t* iterations, double* rel_residual) {
  return solve_host(p, rhs, x, tol, max_iters, restart, iterations, rel_residual, false);
}

BP_API int32_t bp_solve_batch(bp_problem p, const double* rhs, double* x, double tol, int32_t max_iters,
                              int32_t restart, int32_t* iterations, double* rel_residual) {
  if (!iterations || !rel_residual) return fail(BP_ERR_INVALID, "bp_solve_batch: null output array");
  return solve_host(p, rhs, x, tol, max_iters, restart, iterations, rel_residual, true);
}

BP_API int32_t bp_problem_test_wait_timeout(bp_problem p, int32_t enable) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P) return fail(BP_ERR_INVALID, "bp_problem_test_wait_timeout: null problem");
    DeviceGuard g(P->ctx->device);
    if (!fmm_set_stall_test(*P, enable != 0))
      return fail(BP_ERR_UNSUPPORTED, "bp_problem_test_wait_timeout: the problem runs no tensor-core FMM kernel");
    return BP_OK;
  });
}

BP_API int32_t bp_rhs(bp_problem p, const double* charges_xyzq, int32_t n_charges, double eps_solvent, double* rhs) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !rhs || (n_charges > 0 && !charges_xyzq) || n_charges < 0)
      return fail(BP_ERR_INVALID, "bp_rhs: bad argument");
    if (!(eps_solvent > 0)) return fail(BP_ERR_INVALID, "bp_rhs: eps_solvent must be positive");
    if (P->n_scen() > 1)
      return fail(BP_ERR_INVALID, "bp_rhs: a batch problem takes its charges per instance (bp_rhs_posed)");
    DeviceGuard g(P->ctx->device);
    Ctx* c = P->ctx;
    DevBuf& dch = P->scratch_charges;
    const size_t cbytes = sizeof(double) * 4 * (size_t)std::max(1, n_charges);
    if (dch.bytes() < cbytes) dch.alloc(c, cbytes);
    if (n_charges)
      BP_CUDA(cudaMemcpyAsync(dch.get(), charges_xyzq, sizeof(double) * 4 * (size_t)n_charges, cudaMemcpyHostToDevice,
                              c->stream));
    rhs_device(*P, dch.as<double>(), n_charges, eps_solvent, P->d_y.as<double>());
    BP_CUDA(cudaMemcpyAsync(rhs, P->d_y.get(), sizeof(double) * 2 * (size_t)P->n, cudaMemcpyDeviceToHost, c->stream));
    BP_CUDA(cudaStreamSynchronize(c->stream));
    return BP_OK;
  });
}

BP_API int32_t bp_rhs_posed(bp_problem p, const double* const* charges_xyzq, const int32_t* n_charges,
                            double eps_solvent, double* rhs) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !rhs || !charges_xyzq || !n_charges) return fail(BP_ERR_INVALID, "bp_rhs_posed: bad argument");
    if (P->placements.empty())
      return fail(BP_ERR_INVALID, "bp_rhs_posed: the problem was not made by bp_problem_create_posed");
    if (!(eps_solvent > 0)) return fail(BP_ERR_INVALID, "bp_rhs_posed: eps_solvent must be positive");
    for (size_t k = 0; k < P->placements.size(); ++k)
      if (n_charges[k] < 0 || (n_charges[k] > 0 && !charges_xyzq[k]))
        return fail(BP_ERR_INVALID, "bp_rhs_posed: bad charge list of instance " + std::to_string(k));
    DeviceGuard g(P->ctx->device);
    Ctx* c = P->ctx;
    rhs_posed_device(*P, charges_xyzq, n_charges, eps_solvent, P->d_y.as<double>());
    BP_CUDA(cudaMemcpyAsync(rhs, P->d_y.get(), sizeof(double) * 2 * (size_t)P->n, cudaMemcpyDeviceToHost, c->stream));
    BP_CUDA(cudaStreamSynchronize(c->stream));
    return BP_OK;
  });
}

BP_API int32_t bp_energy_coefficients(bp_problem p, int32_t first, int32_t count, const double* charges_xyzq,
                                      int32_t n_charges, double total_area, double* coef_f, double* coef_h) {
  return guarded_engine([&]() -> int32_t {
    Problem* P = as_problem(p);
    if (!P || !coef_f || !coef_h || first < 0 || count <= 0 || first + count > P->n || n_charges < 0 ||
        (n_charges > 0 && !charges_xyzq) || !(total_area > 0))
      return fail(BP_ERR_INVALID, "bp_energy_coefficients: bad argument");
    DeviceGuard g(P->ctx->device);
    Ctx* c = P->ctx;
    DevBuf dch(c, sizeof(double) * 4 * (size_t)std::max(1, n_charges));
    if (n_charges)
      BP_CUDA(cudaMemcpyAsync(dch.get(), charges_xyzq, sizeof(double) * 4 * (size_t)n_charges, cudaMemcpyHostToDevice,
                              c->stream));
    DevBuf out(c, sizeof(double) * 2 * (size_t)count);
    energy_coefficients_device(*P, first, count, dch.as<double>(), n_charges, out.as<double>(),
                               out.as<double>() + count);
    std::vector<double> h(2 * (size_t)count);
    BP_CUDA(cudaMemcpyAsync(h.data(), out.get(), sizeof(double) * 2 * (size_t)count, cudaMemcpyDeviceToHost,
                            c->stream));
    BP_CUDA(cudaStreamSynchronize(c->stream));
    // Gauss-law renormalisation of the f coefficients (host, compensated sums)
    double net = 0.0;
    for (int k = 0; k < n_charges; ++k) net += charges_xyzq[4 * k + 3];
    double total_f = 0.0;
    for (int k = 0; k < count; ++k) total_f -= h[k];
    const double gauss_error = net - total_f;
    for (int k = 0; k < count; ++k) {
      coef_f[k] = h[k] - (P->h_area[first + k] / total_area) * gauss_error;
      coef_h[k] = h[count + k];
    }
    return BP_OK;
  });
}

BP_API int32_t bp_energy(bp_problem p, int32_t first, int32_t count, const double* coef_f, const double* coef_h,
                         double eps_ratio, const double* x, double* energy) {
  Problem* P = as_problem(p);
  if (!P || !coef_f || !coef_h || !x || !energy || first < 0 || count <= 0 || first + count > P->n)
    return fail(BP_ERR_INVALID, "bp_energy: bad argument");
  // Kahan-compensated sum (src/bem/mesh.cpp:1388-1400); 0.5 * N_A e^2 /
  // (eps0 * Angstrom * 1000) converts to kJ/mol (src/bem/constants.h:51).
  const double Avogadro = 6.02214179e23, e = 1.60217646e-19, eps0 = 8.85418782e-12, Ang = 1.0e-10;
  const double conv = Avogadro * e * e / (eps0 * Ang * 1000.0);
  double sum = 0.0, comp = 0.0;
  for (int k = 0; k < count; ++k) {
    const double f = x[first + k], h = x[P->n + first + k];
    const double frag = h * eps_ratio * coef_h[k] - f * coef_f[k];
    const double yv = frag - comp;
    const double t = sum + yv;
    comp = (t - sum) - yv;
    sum = t;
  }
  *energy = sum * 0.5 * conv;
  return BP_OK;
}

}  // extern "C"
