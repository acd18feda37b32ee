// Internal engine types: context, budgeted device buffers, problem state.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <iterator>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.h"
#include "octree.h"

namespace bp {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct BudgetError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct TimeoutError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define BP_CUDA(call)                                                                               \
  do {                                                                                              \
    cudaError_t err__ = (call);                                                                     \
    if (err__ != cudaSuccess)                                                                       \
      throw ::bp::CudaError(std::string(#call) + ": " + cudaGetErrorString(err__) + " @" __FILE__ ":" + \
                            std::to_string(__LINE__));                                              \
  } while (0)

#define BP_LAUNCH_CHECK() BP_CUDA(cudaGetLastError())

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`.  The attribute is process-wide per (device, kernel) while
// problems are created and launched from several threads at once, so the
// limit only ever grows: a problem with a smaller neighbourhood must not
// lower it under another problem's launch.
void ensure_dynamic_smem(const void* kernel, size_t bytes);

template <typename F>
int32_t guarded_engine(F&& f) {
  try {
    return f();
  } catch (const BudgetError& e) {
    return fail(BP_ERR_BUDGET, e.what());
  } catch (const CudaError& e) {
    return fail(BP_ERR_CUDA, e.what());
  } catch (const TimeoutError& e) {
    return fail(BP_ERR_TIMEOUT, e.what());
  } catch (const std::bad_alloc&) {
    return fail(BP_ERR_NOMEM, "host allocation failed");
  } catch (const std::invalid_argument& e) {
    return fail(BP_ERR_INVALID, e.what());
  } catch (const std::exception& e) {
    return fail(BP_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(BP_ERR_INTERNAL, "unknown exception");
  }
}

struct FmmPlan;  // fmm.cu: far-field tables and operators shared by problems

struct Ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;
  uint64_t used = 0;    // bytes of live device buffers
  uint64_t cached = 0;  // bytes of released buffers kept for reuse
  struct Cached {
    void* p;
    uint64_t stamp;  // order of release
  };
  std::multimap<uint64_t, Cached> cache;  // block size -> block
  uint64_t releases = 0;
  std::mutex mu;
  int sm_count = 148;
  // problems and meshes made on the context and not yet deleted: the
  // context may not be destroyed under them
  std::atomic<int> live_problems{0}, live_meshes{0};
  // far-field plans of recent problems, most recently used last
  std::vector<std::shared_ptr<FmmPlan>> fmm_plans;
  std::mutex plan_mu;
  static constexpr size_t kFmmPlans = 4;
  // released blocks beyond this are freed at once, the longest unused first
  static constexpr uint64_t kCacheMax = 16ull << 30;

  // A released block of at least `bytes` (at most a quarter + 1 MB larger),
  // now live, or nullptr.  A problem rebuilt on the same context (a new pose)
  // asks for nearly the same sizes, so it reuses its predecessor's memory
  // without cudaMalloc / cudaFree, which synchronise the whole device.
  void* take(uint64_t bytes, uint64_t& block) {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.lower_bound(bytes);
    if (it == cache.end() || it->first > bytes + bytes / 4 + (1ull << 20)) return nullptr;
    block = it->first;
    void* p = it->second.p;
    cache.erase(it);
    cached -= block;
    used += block;
    return p;
  }
  // Budget for a new block (freeing released blocks first when they stand
  // in the way).
  void charge(uint64_t bytes) {
    std::lock_guard<std::mutex> lk(mu);
    if (budget && used + cached + bytes > budget) trim_locked();
    if (budget && used + bytes > budget)
      throw BudgetError("device allocation of " + std::to_string(bytes) + " bytes exceeds the HBM budget (" +
                        std::to_string(used) + " of " + std::to_string(budget) + " in use)");
    used += bytes;
  }
  void release(uint64_t bytes) {
    std::lock_guard<std::mutex> lk(mu);
    used -= bytes;
  }
  // A live block goes back to the cache.  The context's work is ordered on
  // its stream, so a later user of the block runs after the earlier ones.
  void give(void* p, uint64_t block) {
    std::lock_guard<std::mutex> lk(mu);
    used -= block;
    cache.emplace(block, Cached{p, ++releases});
    cached += block;
    // a problem rebuilt on the context asks for the sizes it released last,
    // so the blocks released longest ago go first
    while (cached > kCacheMax && !cache.empty()) {
      auto oldest = cache.begin();
      for (auto it = cache.begin(); it != cache.end(); ++it)
        if (it->second.stamp < oldest->second.stamp) oldest = it;
      cudaFree(oldest->second.p);
      cached -= oldest->first;
      cache.erase(oldest);
    }
  }
  void trim() {
    std::lock_guard<std::mutex> lk(mu);
    trim_locked();
  }

 private:
  void trim_locked() {
    for (auto& kv : cache) cudaFree(kv.second.p);
    cache.clear();
    cached = 0;
  }
};

// Counts one live object on its context from attach() until destruction.
// Declared as the first member of the object, so it is destroyed last, after
// the object's device buffers have gone back to the context.
struct LiveToken {
  std::atomic<int>* counter = nullptr;
  void attach(std::atomic<int>& c) {
    counter = &c;
    ++c;
  }
  LiveToken() = default;
  LiveToken(const LiveToken&) = delete;
  LiveToken& operator=(const LiveToken&) = delete;
  ~LiveToken() {
    if (counter) --*counter;
  }
};

// Device allocation charged to a context's budget; released on destruction
// (to the context's cache of blocks).
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(Ctx* ctx, size_t bytes) { alloc(ctx, bytes); }
  ~DevBuf() { reset(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { swap(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      swap(o);
    }
    return *this;
  }
  void alloc(Ctx* ctx, size_t bytes) {
    reset();
    if (bytes == 0) return;
    uint64_t block = 0;
    void* p = ctx->take(bytes, block);
    if (!p) {
      ctx->charge(bytes);
      cudaError_t e = cudaMalloc(&p, bytes);
      if (e == cudaErrorMemoryAllocation) {  // released blocks may be in the way
        cudaGetLastError();
        ctx->trim();
        e = cudaMalloc(&p, bytes);
      }
      if (e != cudaSuccess) {
        ctx->release(bytes);
        throw CudaError(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
      }
      block = bytes;
    }
    ctx_ = ctx;
    ptr_ = p;
    bytes_ = bytes;
    block_ = block;
  }
  void reset() {
    if (ptr_) ctx_->give(ptr_, block_);
    ptr_ = nullptr;
    bytes_ = 0;
    block_ = 0;
    ctx_ = nullptr;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr_);
  }
  void* get() const { return ptr_; }
  size_t bytes() const { return bytes_; }

 private:
  void swap(DevBuf& o) {
    std::swap(ctx_, o.ctx_);
    std::swap(ptr_, o.ptr_);
    std::swap(bytes_, o.bytes_);
    std::swap(block_, o.block_);
  }
  Ctx* ctx_ = nullptr;
  void* ptr_ = nullptr;
  size_t bytes_ = 0;   // requested
  uint64_t block_ = 0;  // allocated (a reused block may be larger)
};

template <typename T>
DevBuf upload(Ctx* ctx, const std::vector<T>& v) {
  DevBuf b(ctx, v.size() * sizeof(T));
  if (!v.empty()) BP_CUDA(cudaMemcpyAsync(b.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return b;
}

// Work item of the near-field kernels: a chunk of the rows of one leaf.
struct NfItem {
  int32_t leaf;
  int32_t row_begin;  // offset inside the leaf's row list
  int32_t row_count;
  int32_t qual_total; // qualocation points of those rows (shared-memory sizing)
};

// Near-field block-sparse structure: per leaf a dense |rows| x |cols| block
// of (A, B, C, D) coefficients, rows = the leaf's patches, cols = the
// patches of its 27-box neighbourhood.
struct NearField {
  bool on_demand = false;  // no cached coefficients: instant_kernel every matvec
  bool compact = false;    // FP32 coefficients rounded to 24 bits, 12 bytes a pair
  size_t instant_smem = 0;
  int n_leaves = 0;
  int64_t n_pairs = 0;
  int n_items = 0;
  int max_qual_chunk = 0;
  int max_cols = 0;
  DevBuf rows, row_off, cols, col_off, coef_off, items;
  DevBuf coef;  // 4 * n_pairs of float or double; compact: 2 * n_pairs + n_pairs words
  std::vector<int64_t> h_row_off, h_col_off, h_coef_off;
  std::vector<int32_t> h_rows, h_cols;
  std::vector<NfItem> h_items;
};

// A mesh's node patches in its own frame, checked and uploaded once
// (bp_mesh_create); instances of it are placed on the device.
struct DevMesh {
  LiveToken live;  // first member: destroyed last
  Ctx* ctx = nullptr;
  int n = 0;
  double centre[3] = {0, 0, 0};
  std::vector<double> h_centroid, h_normal, h_area, h_gc;
  std::vector<int32_t> h_qual_off, h_quad_off, h_gal_off;
  int n_qual_pts = 0, n_quad_pts = 0, n_gal_pts = 0;
  DevBuf d_qual, d_quad, d_gal;  // SoA of double, 7 arrays each
  // potential of a charge list given in the mesh's frame at the mesh's
  // qualocation points (2 doubles per point), kept for rigid moves
  struct SelfPotential {
    std::vector<double> charges;  // x, y, z, q in the mesh's frame
    double scale = 0;
    bool fp64 = true;
    DevBuf vals;
  };
  std::vector<SelfPotential> self_potential;  // most recently used last
  static constexpr size_t kSelfPotentials = 4;
  // Near-field coefficients of the mesh's own patch pairs closer than
  // `radius` (centroid distance), computed once in the mesh's frame: a rigid
  // move leaves them unchanged, so every posed problem with this mesh and
  // kappa looks them up instead of integrating them (mixed engine, meshes
  // with one quadrature point per patch).  Per pair six FP32 parts (A, Bu,
  // Bg, Cg, Cu, D): B = Bu - Bg / eps, C = Cg - Cu / eps, D / eps for the
  // instance's dielectric ratio eps.
  struct PairCache {
    double kappa = -1;
    float radius = 0;
    int64_t n_pairs = 0;
    int max_row = 0;  // longest partner list
    DevBuf off;   // int64 [n + 1]
    DevBuf js;    // int32 [n_pairs]: the partners of each patch, ascending
    DevBuf vals;  // float [n_pairs][6]
  };
  PairCache pair_cache;
  // posed problems placed from this mesh keep it: bp_mesh_destroy while any
  // exists leaves the deletion to the last of them
  int users = 0;
  bool destroy_pending = false;
  std::mutex mu;
};

inline void mesh_acquire(DevMesh* m) {
  std::lock_guard<std::mutex> lk(m->mu);
  ++m->users;
}
// True when the caller must delete the mesh (its destruction was asked for
// and this was its last user).
inline bool mesh_release(DevMesh* m) {
  std::lock_guard<std::mutex> lk(m->mu);
  return --m->users == 0 && m->destroy_pending;
}

// Where an instance of a device-resident mesh sits in a posed problem:
// p -> R (p - c) + o, its qualocation points at [q_begin, q_begin + q_count).
struct Placement {
  DevMesh* mesh = nullptr;
  double R[9], c[3], o[3];
  int q_begin = 0, q_count = 0;
  int scenario = 0;  // the independent scenario of a batch the instance belongs to
};

struct Problem;
struct FmmState;  // far-field state (fmm.cu)
void fmm_destroy(FmmState*);

struct Problem {
  LiveToken live;  // first member: destroyed last
  Ctx* ctx = nullptr;
  int n = 0;
  bp_params params{};
  bool fp64 = true;
  TreeInfo tree;
  std::vector<Placement> placements;  // set by bp_problem_create_posed / _batch
  // Independent scenarios (bp_problem_create_batch): scenario s owns patches
  // [scen_first[s], scen_first[s+1]), has its own tree in the cube of centre
  // scen_centre[3s..3s+2] (all of edge params.cube_edge) and its own GMRES;
  // no interaction crosses scenarios.  An ordinary problem is one scenario.
  std::vector<int> scen_first;
  std::vector<double> scen_centre;
  int n_scen() const { return (int)scen_first.size() - 1; }
  // patches (original order)
  std::vector<double> h_centroid, h_normal, h_area, h_eps, h_gc;
  std::vector<int32_t> h_qual_off, h_quad_off, h_gal_off;
  int n_qual_pts = 0, n_quad_pts = 0, n_gal_pts = 0;  // point counts of the device point lists
  DevBuf d_centroid, d_normal, d_area, d_eps;               // double
  DevBuf d_qual_off, d_quad_off, d_gal_off;                 // int32
  DevBuf d_qual, d_quad, d_gal;                             // SoA of double, 7 arrays
  DevBuf d_qual_f, d_quad_f;                                // SoA of float (mixed)
  DevBuf d_inst_of;  // int32 [n]: the placement of each patch (pair-cache lookups)
  DevBuf d_diag;                                            // 4n double (singular + corrections)
  NearField nf;
  std::unique_ptr<FmmState, void (*)(FmmState*)> fmm{nullptr, fmm_destroy};
  DevBuf fmm_contents;  // node-major patch lists of the tree (int32)
  // matvec scratch
  DevBuf d_x, d_y;  // 2n double each
  DevBuf d_yfar;    // 2n double: far field, added to the near field at the end
  // graph of one matvec (d_gx -> d_gy): near field on the main stream and the
  // FMM on a side stream, joined before the final add
  DevBuf d_gx, d_gy;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool graph_failed = false;
  int* h_status = nullptr;  // pinned host word: the far field's status read back behind a result
  // Krylov workspace
  DevBuf d_V, d_w, d_scal, d_seg;
  // one GMRES cycle's Arnoldi loop as a graph with a device-side WHILE node
  // (built for basis size gmres_graph_m on the V / scalar blocks it was
  // captured with)
  cudaGraphExec_t gmres_graph = nullptr;
  int gmres_graph_m = 0;
  const void* gmres_graph_v = nullptr;
  bool gmres_graph_failed = false;
  // grow-only scratch of the source terms (charges, per-point values, the
  // right-hand side of bp_solve): kept so repeated calls allocate nothing
  DevBuf scratch_charges, scratch_vals, scratch_b;
  // qualocation point indices in spatial order within each instance's range
  // (patches in the tree's leaf order), for the mixed right-hand side; made
  // on its first use
  DevBuf d_qual_order;
  int krylov_m = 0;
  double tree_ms = 0, assemble_ms = 0, fmm_setup_ms = 0, setup_ms = 0;
  // the near-field assembly runs on a stream of its own while the far field
  // is set up; its inputs stay allocated until it is joined (nf_join)
  cudaStream_t asm_stream = nullptr;
  cudaEvent_t asm_in = nullptr, asm_t0 = nullptr, asm_t1 = nullptr;
  DevBuf asm_gc, asm_items, asm_views;
  ~Problem() {
    if (asm_stream) {
      cudaStreamSynchronize(asm_stream);
      cudaStreamDestroy(asm_stream);
    }
    if (asm_in) cudaEventDestroy(asm_in);
    if (asm_t0) cudaEventDestroy(asm_t0);
    if (asm_t1) cudaEventDestroy(asm_t1);
    for (const Placement& pl : placements)
      if (mesh_release(pl.mesh)) delete pl.mesh;
    if (graph) cudaGraphExecDestroy(graph);
    if (gmres_graph) cudaGraphExecDestroy(gmres_graph);
    if (h_status) cudaFreeHost(h_status);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
  }
};

// Optional per-stage timing of a matvec with CUDA events on the stream.
constexpr int kStages = 8;  // near(+add), P2M, M2M, M->X, X->L (translations + conversion), L2P prep, L2L, L2P eval
struct StageTimes {
  struct Rec {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  int launches[kStages] = {0, 0, 0, 0, 0, 0, 0, 0};
  cudaStream_t stream = nullptr;
  int open_stage = -1;
  cudaEvent_t open_ev = nullptr, close_ev = nullptr;
  // both events are created before the first is recorded, so no host-side
  // event creation falls inside the measured interval
  void begin(int s, cudaStream_t st) {
    stream = st;
    open_stage = s;
    BP_CUDA(cudaEventCreate(&open_ev));
    BP_CUDA(cudaEventCreate(&close_ev));
    BP_CUDA(cudaEventRecord(open_ev, st));
  }
  void end(int launches_in_stage) {
    BP_CUDA(cudaEventRecord(close_ev, stream));
    recs.push_back({open_stage, open_ev, close_ev});
    launches[open_stage] += launches_in_stage;
    open_ev = close_ev = nullptr;
  }
  double ms(int s) const {
    double t = 0;
    for (const Rec& r : recs)
      if (r.stage == s) {
        float f = 0;
        cudaEventElapsedTime(&f, r.a, r.b);
        t += f;
      }
    return t;
  }
  ~StageTimes() {
    for (Rec& r : recs) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
  }
};

// device_tree.cu: leaf-capped octree of the n centroids (device, xyz
// interleaved) in the cube (centre, edge); at most `cap` patches per leaf
void build_device_tree(Ctx* c, const double* d_centroids, int n, const double centre[3], double edge, int cap,
                       TreeInfo& out);
// nearfield.cu
void nf_build_structure(Problem& P);
void nf_assemble(Problem& P);  // launches the assembly on P.asm_stream
void nf_join(Problem& P);      // orders the context's stream after it
// y = near field (incl. singular diagonal) of x, plus yfar if not null;
// returns the number of kernel launches (0 when the problem has no near-field
// items, in which case y is not written)
int nf_apply(Problem& P, const double* x_dev, double* y_dev, const double* yfar_dev, cudaStream_t stream);
// fmm.cu
bool fmm_active(const Problem& P);
struct FmmWork {
  long long m2x_cols = 0, x2l_cols = 0, xl_entries = 0, shift_cols = 0;
  int plane_waves = 0, coefficients = 0;  // per direction / per channel
};
FmmWork fmm_work(const Problem& P);
// Throws TimeoutError if a tensor-core FMM kernel of this problem gave up on
// a bounded wait since the problem was created (its results are then void).
// Synchronises the context stream.
void fmm_check_waits(Problem& P);
// The same check split in two: the device word to copy back behind the
// caller's last copy (null without a tensor-core far field), then the
// value read, raising TimeoutError (and clearing the word) when set.
const int* fmm_status_dev(Problem& P);
void fmm_raise_if(Problem& P, int flag);
// Timeout test switch of the tensor-core FMM kernels (see
// bp_problem_test_wait_timeout); false when the problem has none.
bool fmm_set_stall_test(Problem& P, bool on);
void fmm_setup(Problem& P);
void fmm_apply(Problem& P, const double* x_dev, double* y_dev, StageTimes* st, cudaStream_t stream);
void matvec_setup(Problem& P);
// krylov.cu
void matvec_device(Problem& P, const double* x_dev, double* y_dev, StageTimes* st = nullptr);
// GMRES of every scenario of P (one for an ordinary problem): rel_resid and
// iters (may be null) receive one entry per scenario; returns the most
// iterations any scenario took.  x_is_zero: the caller knows x = 0 on entry,
// so the first residual is -b without a matvec.
int gmres_device(Problem& P, const double* b_dev, double* x_dev, double tol, int max_iters, int restart,
                 double* rel_resid, int* iters = nullptr, bool x_is_zero = false);
// true when every entry of the device vector is zero (one reduction, synchronises)
bool device_all_zero(Problem& P, const double* x_dev, int64_t len);
// sources.cu
void rhs_device(Problem& P, const double* charges_dev, int n_charges, double eps_solvent, double* rhs_dev);
// right-hand side of a posed problem from each instance's charges in its
// mesh's frame (host arrays); own-charge potentials cached on the meshes
void rhs_posed_device(Problem& P, const double* const* charges_host, const int32_t* n_charges, double eps_solvent,
                      double* rhs_dev);
void energy_coefficients_device(Problem& P, int first, int count, const double* charges_dev, int n_charges,
                                double* cf_dev, double* ch_dev);

}  // namespace bp
