// mpm_gpu.cu -- C ABI (include/mpm_gpu.h): solver handle, host-side set-up
// that mirrors the reference's MPMBase initialisation, device buffers and the
// step loop.
#include <cuda_runtime.h>
#include <sched.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <type_traits>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpm_gpu.h"
#include "json_lite.hpp"
#include "mpm_kernels.h"
#include "mpm_math.cuh"
#include "mpm_state.cuh"

using namespace mpm_b200;

#define MPM_VERSION "mpm_b200 0.1.0 (sm_100a)"

namespace {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct InvalidArg : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free();
    if (count == 0) return;
    ck(cudaMalloc(&p, sizeof(T) * count), "cudaMalloc");
    n = count;
  }
  // keeps the allocation when it already holds exactly count elements
  void resize(size_t count) {
    if (count != n || (count && !p)) alloc(count);
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T* h, size_t count, cudaStream_t st) {
    if (count > n) alloc(count);
    if (count) ck(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, st), "H2D");
  }
  void download(T* h, size_t count, cudaStream_t st) const {
    if (count) ck(cudaMemcpyAsync(h, p, sizeof(T) * count, cudaMemcpyDeviceToHost, st), "D2H");
  }
  ~DevBuf() { free(); }
};

struct HostBC {
  std::map<unsigned, double> vel, acc;  // ascending direction (node.tcc std::map)
  bool friction = false;
  unsigned fdir = 0;
  int fsign = 0;
  double mu = 0;
  bool rotated = false;  // general boundary: constraints in the frame of these angles
  double angles[3] = {0, 0, 0};
};

// Host worker threads kept for the life of the process, for the per-particle
// conversions between the caller's rows and the device layout and the staged
// copies through pinned memory: a parallel_for wakes them instead of starting
// threads (the staged copies call it once per 64 MiB chunk).  One job runs at a
// time; a call made while a job runs (another handle's thread, or a nested
// call from a worker) runs on its own thread.
class HostPool {
 public:
  static HostPool& get() {
    static HostPool pool;
    return pool;
  }
  int64_t threads() const { return (int64_t)workers_.size() + 1; }
  // false when the pool is busy: the caller runs the job itself
  template <class Job>
  bool run(int64_t ntasks, Job& job) {
    std::unique_lock<std::mutex> busy(busy_, std::try_to_lock);
    if (!busy.owns_lock() || in_worker()) return false;
    {
      std::lock_guard<std::mutex> g(mu_);
      task_ = [&job](int64_t t) { job(t); };
      ntasks_ = ntasks;
      next_ = 1;  // task 0 runs on the calling thread
      done_ = 0;
      ++gen_;
    }
    cv_.notify_all();
    job(0);
    finish_one();
    std::unique_lock<std::mutex> g(mu_);
    all_done_.wait(g, [&] { return done_ == ntasks_; });
    task_ = nullptr;
    return true;
  }

 private:
  HostPool() {
    int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
    cpu_set_t set;  // the CPUs this process may run on, when fewer
    if (sched_getaffinity(0, sizeof(set), &set) == 0) hw = std::min<int64_t>(hw, CPU_COUNT(&set));
    hw = std::max<int64_t>(1, hw);
    for (int64_t w = 1; w < hw; ++w) workers_.emplace_back([this] { loop(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  static bool& in_worker() {
    static thread_local bool w = false;
    return w;
  }
  void finish_one() {
    std::lock_guard<std::mutex> g(mu_);
    if (++done_ == ntasks_) all_done_.notify_all();
  }
  void loop() {
    in_worker() = true;
    uint64_t seen = 0;
    std::unique_lock<std::mutex> g(mu_);
    for (;;) {
      cv_.wait(g, [&] { return stop_ || (gen_ != seen && next_ < ntasks_); });
      if (stop_) return;
      while (next_ < ntasks_) {
        const int64_t t = next_++;
        auto task = task_;
        g.unlock();
        task(t);
        g.lock();
        if (++done_ == ntasks_) all_done_.notify_all();
      }
      seen = gen_;
    }
  }
  std::vector<std::thread> workers_;
  std::mutex busy_, mu_;
  std::condition_variable cv_, all_done_;
  std::function<void(int64_t)> task_;
  int64_t ntasks_ = 0, next_ = 0, done_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// f(a, b) over [0, n) split across the host's threads (at least 32768 items a
// thread); the first exception a worker throws is rethrown here.
template <class F>
void parallel_for(int64_t n, F f) {
  HostPool& pool = HostPool::get();
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(pool.threads(), n / 32768));
  if (nt == 1) {
    f((int64_t)0, n);
    return;
  }
  std::exception_ptr err;
  std::mutex mu;
  auto job = [&](int64_t w) {
    try {
      f(n * w / nt, n * (w + 1) / nt);
    } catch (...) {
      std::lock_guard<std::mutex> g(mu);
      if (!err) err = std::current_exception();
    }
  };
  if (!pool.run(nt, job))
    for (int64_t w = 0; w < nt; ++w) job(w);
  if (err) std::rethrow_exception(err);
}

}  // namespace

namespace mpm_b200 {

const char* kernel_name(int kid) {
  static const char* names[K_NKERNELS] = {"sort",  "p2g",   "nodes_velocity", "stress",
                                          "p2g_forces", "nodes_acceleration", "g2p",
                                          "mc_return", "locate_fallback",
                                          "adjoint_recompute", "adjoint_material",
                                          "adjoint_return", "adjoint_kinematics",
                                          "adjoint_scatter", "adjoint_nodes", "adjoint_p2g"};
  return (kid >= 0 && kid < K_NKERNELS) ? names[kid] : "?";
}

struct ProfilerImpl {
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  cudaEvent_t open_start = nullptr;
  cudaEvent_t take() {
    if (pool.empty()) {
      cudaEvent_t e;
      ck(cudaEventCreate(&e), "cudaEventCreate");
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
};

void Profiler::begin(int kid, cudaStream_t st, int kernels) {
  (void)kid;
  launches += kernels;
  if (!enabled) return;
  if (!impl) impl = new ProfilerImpl();
  auto* P = static_cast<ProfilerImpl*>(impl);
  P->open_start = P->take();
  ck(cudaEventRecord(P->open_start, st), "cudaEventRecord");
}

void Profiler::end(int kid, cudaStream_t st) {
  if (!enabled) return;
  auto* P = static_cast<ProfilerImpl*>(impl);
  cudaEvent_t e = P->take();
  ck(cudaEventRecord(e, st), "cudaEventRecord");
  P->pending.push_back({kid, {P->open_start, e}});
}

void Profiler::collect() {
  if (!impl) return;
  auto* P = static_cast<ProfilerImpl*>(impl);
  for (auto& r : P->pending) {
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, r.second.first, r.second.second), "cudaEventElapsedTime");
    total_ms[r.first] += ms;
    count[r.first] += 1;
    P->pool.push_back(r.second.first);
    P->pool.push_back(r.second.second);
  }
  P->pending.clear();
}

void Profiler::reset() {
  collect();
  launches = 0;
  for (int k = 0; k < K_NKERNELS; ++k) {
    total_ms[k] = 0;
    count[k] = 0;
  }
}

Profiler::~Profiler() {
  if (!impl) return;
  auto* P = static_cast<ProfilerImpl*>(impl);
  for (auto e : P->pool) cudaEventDestroy(e);
  for (auto& r : P->pending) {
    cudaEventDestroy(r.second.first);
    cudaEventDestroy(r.second.second);
  }
  delete P;
}

}  // namespace mpm_b200

// The adjoint's record of a forward run: the particle state every `every`
// steps (checkpoints), room for the states of one segment between two
// checkpoints (recomputed during the reverse sweep), the end state, and the
// reverse sweep's work arrays.
struct AdjointTape {
  bool recorded = false;
  int64_t nsteps = 0, every = 0, step0 = 0, np = 0;
  int nparams = 0;
  size_t pf_n = 0, sv_n = 0, cell_n = 0;  // elements of one stored state
  // Checkpoints and segment states keep only the particle rows the recompute
  // and the reverse kernels read -- x, v, stress, volume, density, mass --
  // not u, strain and F, which no later position, velocity or stress depends
  // on; the run's end state is kept whole.  Row ranges [first, last) of the
  // FP64 particle buffer, in units of npad.
  int nranges = 0;
  int range[3][2] = {};
  size_t pfc_n = 0;  // elements of one compact particle state
  DevBuf<double> ck_pf, ck_sv, seg_pf, seg_sv, fin_pf, fin_sv;
  DevBuf<int32_t> ck_cell, seg_cell, fin_cell;
  DevBuf<double> adj, deps, dsbar, coef, theta, apart, nbar, sv_seed;
  DevBuf<unsigned char> mats_zero, mats_param;
  double mass_floor = 0.0;
};

struct mpm_gpu_solver {
  mpm_gpu_config cfg{};
  int dim = 3, nv = 8;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t step = 0;
  bool mesh_set = false, initialised = false;

  // mesh (host)
  int64_t nnodes = 0, ncells = 0;
  std::vector<double> coords;           // nnodes*dim
  std::vector<int32_t> cell_nodes;      // ncells*nv
  std::vector<CellGeom> geom;           // ncells
  std::vector<double> cell_volume;      // ncells
  std::vector<int32_t> nb_off, nb;      // neighbour CSR
  std::vector<int32_t> bin_off, bin_cells;
  double bmin[3] = {0, 0, 0}, bsize[3] = {1, 1, 1};
  int32_t bn[3] = {1, 1, 1};
  std::map<int64_t, HostBC> bcs;        // node id -> constraints
  bool structured = false;
  bool isoparametric = false;  // general cells: isoparametric local coordinates
  int32_t gcells[3] = {1, 1, 1};
  std::vector<double> axis[3];
  std::vector<double> axis_ihl[3];  // 2 / (axis[i + 1] - axis[i]): J^-1 of the box cells

  // materials
  std::vector<MaterialParams> mats;
  std::map<int32_t, int> mat_index;     // material id -> slot

  // particles (host staging).  On the device every particle field is an
  // array of npad = np rounded up to a multiple of PAD_PARTICLES entries; the
  // padding rows are removed particles (cell -1), so a block's slice of a
  // field is one aligned contiguous segment.
  int64_t np = 0;
  int64_t npad = 0;
  std::vector<double> p_coords;         // np*dim (creation)
  std::vector<uint16_t> p_mat;
  std::map<int64_t, std::map<unsigned, double>> p_vc;  // velocity constraints of constrained particles
  bool p_vc_dirty = false;

  // device
  DevState ds;
  DevBuf<double> d_pf, d_sv, d_nf, d_ncoord, d_xnext, d_mapb;
  DevBuf<int32_t> d_cell, d_bc_index, d_cell_nodes, d_nb_off, d_nb, d_bin_off, d_bin_cells, d_lost;
  DevBuf<uint16_t> d_mat;
  DevBuf<uint8_t> d_active;
  DevBuf<int16_t> d_pvc;
  DevBuf<CellGeom> d_geom;
  DevBuf<unsigned> d_words;  // [0] nlost, [1] err, [2] nplastic, [3] nplastic_heavy, [4, 6) grid barrier,
                             // [6, 8) the persistent launches' step counter (int64)
  DevBuf<int32_t> d_plist;
  DevBuf<double> d_pbuf;
  DevBuf<uint8_t> d_rpass;
  DevBuf<MaterialParams> d_mats;
  DevBuf<double> d_axis[3];
  DevBuf<double> d_axis_ihl[3];
  DevBuf<double> d_dndx_c, d_partials;
  DevBuf<int32_t> d_nc_off, d_nc_cell, d_cnt, d_start, d_rank, d_order, d_bsum;
  DevBuf<int8_t> d_nc_slot;
  std::vector<double> dndx_c;                 // [ncells][nv][dim]
  std::vector<int32_t> nc_off, nc_cell;       // node -> cells (general meshes)
  std::vector<int8_t> nc_slot;
  DevBuf<NodeBC> d_bcs;
  DevBuf<ParticleVC> d_pvcs;
  bool any_mc = false;
  Profiler prof;

  // per-particle data the step never changes, kept for the PODParticle
  // records: id, natural size [3][np], acceleration [3][np]
  std::vector<uint64_t> p_id;
  std::vector<double> p_nsize, p_acc;
  bool aux_dirty = true;
  DevBuf<uint64_t> d_pid;
  DevBuf<double> d_nsize, d_pacc;
  DevBuf<int32_t> d_matid, d_list;
  DevBuf<uint32_t> d_nstate;
  DevBuf<uint8_t> d_stage;
  DevBuf<double> d_rows;  // the caller's particle rows, staged for the device conversion
  uint8_t* h_stage = nullptr;  // pinned, two halves
  double* h_rows = nullptr;    // pinned copy of the staged particle rows
  size_t h_rows_n = 0;
  size_t h_stage_bytes = 0;
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};

  // launch shape of the value steps (mpm_gpu_set_launch_shape, mpm_gpu_autotune);
  // zeros are the built-in defaults
  int shape_p2g_tile = 0, shape_node_threads = 0, shape_return_bps = 0;
  int persistent_steps = 0;  // > 0: steps per persistent launch
  // one captured step, replayed while the device state and step arguments
  // stay the same
  cudaGraphExec_t graph = nullptr;
  // the persistent launch of persistent_steps steps, captured (its state, arguments)
  cudaGraphExec_t pgraph = nullptr;
  DevState pgraph_state{};
  StepArgs pgraph_args{};
  int64_t pgraph_steps = 0;
  bool pgraph_ok = true;
  DevState graph_state{};
  StepArgs graph_args{};
  int64_t graph_launches = 0;
  bool graph_ok = true;

  // sensitivities: tangent buffers (layouts of pf, sv, nf, partials)
  int ntangent = 0;
  double tangent_mass_floor = 0.0;
  DevBuf<double> d_pft[MAX_TANGENTS], d_svt[MAX_TANGENTS], d_nft[MAX_TANGENTS],
      d_partt[MAX_TANGENTS];
  DevBuf<unsigned char> d_mats_t;
  DevBuf<double> d_tpbuf;
  std::unique_ptr<AdjointTape> tape;  // reverse-mode adjoint (mpm_gpu_adjoint_record)

  // mixed precision: d_pf holds [x, u, pdstrain] in FP64, the rest is FP32
  bool mixed = false;
  DevBuf<float> d_pm, d_svf, d_nfv, d_partials_f, d_dndx_cf;
  DevBuf<MaterialT<float>> d_mats_f;

  int nfields() const { return dim == 2 ? PF<2>::NF : PF<3>::NF; }
  void set_np(int64_t n) {
    np = n;
    npad = (n + PAD_PARTICLES - 1) / PAD_PARTICLES * PAD_PARTICLES;
  }
  int nfields_x() const { return dim == 2 ? PDX<2>::ND : PDX<3>::ND; }
  int nfields_m() const { return dim == 2 ? PM<2>::NF : PM<3>::NF; }
  int nnf() const { return dim == 2 ? NF<2>::NNF : NF<3>::NNF; }
};

namespace {

int fail(mpm_gpu_t h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

double norm_d(int dim, const double* a) {
  double s = a[0] * a[0];
  for (int i = 1; i < dim; ++i) s = s + a[i] * a[i];
  return std::sqrt(s);
}

// cell.tcc:255-279 (centroid, mean length), :458-463 / :566-571 (local
// coordinate lengths); quadrilateral_element.tcc:473-496 and
// hexahedron_element.tcc:559-596 (volume)
void cell_geometry(int dim, const double* X, CellGeom* g, double* volume) {
  const int nv = dim == 2 ? 4 : 8;
  for (int i = 0; i < 3; ++i) g->centroid[i] = g->len[i] = 0.;
  for (int n = 0; n < nv; ++n)
    for (int i = 0; i < dim; ++i) g->centroid[i] = g->centroid[i] + X[n * dim + i];
  for (int i = 0; i < dim; ++i) g->centroid[i] = g->centroid[i] / nv;
  static const int q4s[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  static const int h8s[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                 {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  const int ns = dim == 2 ? 4 : 12;
  double ml = 0.;
  for (int s = 0; s < ns; ++s) {
    const int a = dim == 2 ? q4s[s][0] : h8s[s][0];
    const int b = dim == 2 ? q4s[s][1] : h8s[s][1];
    double d[3];
    for (int i = 0; i < dim; ++i) d[i] = X[a * dim + i] - X[b * dim + i];
    ml += norm_d(dim, d);
  }
  g->mean_length = ml / ns;
  double d[3];
  for (int i = 0; i < dim; ++i) d[i] = X[0 * dim + i] - X[1 * dim + i];
  g->len[0] = norm_d(dim, d);
  for (int i = 0; i < dim; ++i) d[i] = X[1 * dim + i] - X[2 * dim + i];
  g->len[1] = norm_d(dim, d);
  if (dim == 3) {
    for (int i = 0; i < dim; ++i) d[i] = X[1 * dim + i] - X[5 * dim + i];
    g->len[2] = norm_d(dim, d);
  }
  if (dim == 2) {
    auto len = [&](int a, int b) {
      double e[2] = {X[a * 2] - X[b * 2], X[a * 2 + 1] - X[b * 2 + 1]};
      return norm_d(2, e);
    };
    const double a = len(0, 3), b = len(2, 3), c = len(1, 2), dd = len(0, 1);
    const double p = len(0, 2), q = len(1, 3);
    *volume = 0.25 * std::sqrt(4 * p * p * q * q - std::pow((a * a + c * c - b * b - dd * dd), 2.0));
  } else {
    auto row = [&](int n, double* r) { for (int i = 0; i < 3; ++i) r[i] = X[n * 3 + i]; };
    auto sub = [](const double* x, const double* y, double* r) { for (int i = 0; i < 3; ++i) r[i] = x[i] - y[i]; };
    auto add = [](const double* x, const double* y, double* r) { for (int i = 0; i < 3; ++i) r[i] = x[i] + y[i]; };
    auto cross = [](const double* x, const double* y, double* r) {
      r[0] = x[1] * y[2] - x[2] * y[1];
      r[1] = x[2] * y[0] - x[0] * y[2];
      r[2] = x[0] * y[1] - x[1] * y[0];
    };
    auto dot = [](const double* x, const double* y) { return (x[0] * y[0] + x[1] * y[1]) + x[2] * y[2]; };
    double A[3], B[3], C[3], D[3], E[3], F[3], G[3], H[3];
    row(7, A); row(6, B); row(2, C); row(3, D); row(4, E); row(5, F); row(1, G); row(0, H);
    double t1[3], t2[3], bd[3], eb[3], de[3], x1[3], s1[3], s2[3], s3[3], s4[3], tmp[3];
    sub(B, D, t1); sub(C, A, t2); cross(t1, t2, bd);
    sub(E, B, t1); sub(F, A, t2); cross(t1, t2, eb);
    sub(D, E, t1); sub(H, A, t2); cross(t1, t2, de);
    add(bd, eb, tmp); add(tmp, de, s1);
    sub(C, G, t1); sub(C, F, t2); cross(t1, t2, x1); add(bd, x1, s2);
    sub(F, G, t1); sub(H, F, t2); cross(t1, t2, x1); add(eb, x1, s3);
    sub(H, G, t1); sub(H, C, t2); cross(t1, t2, x1); add(de, x1, s4);
    double ag[3], bg[3], eg[3], dg[3];
    sub(A, G, ag); sub(B, G, bg); sub(E, G, eg); sub(D, G, dg);
    *volume = (1.0 / 12) * dot(ag, s1) + (1.0 / 12) * dot(bg, s2) + (1.0 / 12) * dot(eg, s3) +
              (1.0 / 12) * dot(dg, s4);
  }
}

void build_bins(mpm_gpu_t h) {
  const int dim = h->dim;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  double maxr = 0;
  for (int64_t c = 0; c < h->ncells; ++c) {
    const CellGeom& g = h->geom[c];
    const double r = 2. * g.mean_length;
    maxr = std::max(maxr, r);
    for (int i = 0; i < dim; ++i) {
      lo[i] = std::min(lo[i], g.centroid[i] - r);
      hi[i] = std::max(hi[i], g.centroid[i] + r);
    }
  }
  double extent = 0;
  for (int i = 0; i < dim; ++i) extent = std::max(extent, hi[i] - lo[i]);
  // widen every range by far more than the rounding of the bin arithmetic
  const double pad = 1e-9 * std::max(extent, 1e-300);
  int64_t total = 1;
  for (int i = 0; i < 3; ++i) {
    if (i >= dim) {
      h->bn[i] = 1;
      h->bmin[i] = 0;
      h->bsize[i] = 1;
      continue;
    }
    h->bmin[i] = lo[i] - 2 * pad;
    h->bsize[i] = std::max(2. * maxr, 1e-300);
    h->bn[i] = (int32_t)std::max<int64_t>(1, (int64_t)std::ceil((hi[i] + 2 * pad - h->bmin[i]) / h->bsize[i]) + 1);
    total *= h->bn[i];
  }
  std::vector<std::vector<int32_t>> bins(total);
  for (int64_t id = 0; id < h->ncells; ++id) {
    const CellGeom& g = h->geom[id];
    const double r = 2. * g.mean_length;
    int64_t b0[3] = {0, 0, 0}, b1[3] = {0, 0, 0};
    for (int i = 0; i < dim; ++i) {
      b0[i] = std::max<int64_t>(0, (int64_t)std::floor((g.centroid[i] - r - pad - h->bmin[i]) / h->bsize[i]));
      b1[i] = std::min<int64_t>(h->bn[i] - 1, (int64_t)std::floor((g.centroid[i] + r + pad - h->bmin[i]) / h->bsize[i]));
    }
    for (int64_t k = b0[2]; k <= b1[2]; ++k)
      for (int64_t j = b0[1]; j <= b1[1]; ++j)
        for (int64_t i = b0[0]; i <= b1[0]; ++i)
          bins[(k * h->bn[1] + j) * h->bn[0] + i].push_back((int32_t)id);
  }
  h->bin_off.assign(total + 1, 0);
  for (int64_t b = 0; b < total; ++b) h->bin_off[b + 1] = h->bin_off[b] + (int32_t)bins[b].size();
  h->bin_cells.resize(h->bin_off[total]);
  for (int64_t b = 0; b < total; ++b)
    std::copy(bins[b].begin(), bins[b].end(), h->bin_cells.begin() + h->bin_off[b]);
}

// Recognise a tensor-product grid: node (i,j,k) = i + nx*(j + ny*k) sits at
// (ax[i], ay[j], az[k]) with strictly increasing axes, and cell
// (i,j,k) = i + cx*(j + cy*k) has the reference node order.
bool detect_structured(mpm_gpu_t h) {
  const int dim = h->dim;
  const double* X = h->coords.data();
  int64_t n[3] = {1, 1, 1};
  // count nodes along x: until the y coordinate changes
  int64_t stride = 1;
  for (int d = 0; d < dim; ++d) {
    int64_t c = 1;
    while (stride * (c + 1) <= h->nnodes) {
      bool same_other = true;
      for (int e = 0; e < dim; ++e)
        if (e != d && X[(stride * c) * dim + e] != X[0 * dim + e]) same_other = false;
      if (!same_other || !(X[(stride * c) * dim + d] > X[(stride * (c - 1)) * dim + d])) break;
      ++c;
    }
    n[d] = c;
    stride *= c;
  }
  if (stride != h->nnodes) return false;
  for (int d = 0; d < dim; ++d)
    if (n[d] < 2) return false;
  std::vector<double> ax[3];
  int64_t st[3] = {1, n[0], n[0] * n[1]};
  for (int d = 0; d < dim; ++d) {
    ax[d].resize(n[d]);
    for (int64_t i = 0; i < n[d]; ++i) ax[d][i] = X[(i * st[d]) * dim + d];
  }
  for (int64_t id = 0; id < h->nnodes; ++id) {
    int64_t r = id;
    for (int d = 0; d < dim; ++d) {
      const int64_t i = r % n[d];
      r /= n[d];
      if (X[id * dim + d] != ax[d][i]) return false;
    }
  }
  const int64_t cx = n[0] - 1, cy = n[1] - 1, cz = dim == 3 ? n[2] - 1 : 1;
  if (cx * cy * cz != h->ncells) return false;
  for (int64_t c = 0; c < h->ncells; ++c) {
    const int64_t i = c % cx, j = (c / cx) % cy, k = c / (cx * cy);
    auto nid = [&](int64_t a, int64_t b, int64_t e) { return a + n[0] * (b + n[1] * e); };
    const int32_t* cn = &h->cell_nodes[c * h->nv];
    if (dim == 2) {
      const int64_t ref[4] = {nid(i, j, 0), nid(i + 1, j, 0), nid(i + 1, j + 1, 0), nid(i, j + 1, 0)};
      for (int q = 0; q < 4; ++q)
        if (cn[q] != ref[q]) return false;
    } else {
      const int64_t ref[8] = {nid(i, j, k),         nid(i + 1, j, k),     nid(i + 1, j + 1, k),
                              nid(i, j + 1, k),     nid(i, j, k + 1),     nid(i + 1, j, k + 1),
                              nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)};
      for (int q = 0; q < 8; ++q)
        if (cn[q] != ref[q]) return false;
    }
  }
  h->gcells[0] = (int32_t)cx;
  h->gcells[1] = (int32_t)cy;
  h->gcells[2] = (int32_t)cz;
  for (int d = 0; d < 3; ++d) {
    h->axis[d] = d < dim ? ax[d] : std::vector<double>{0.0, 1.0};
    const std::vector<double>& a = h->axis[d];
    h->axis_ihl[d].resize(a.size() - 1);
    for (size_t i = 0; i + 1 < a.size(); ++i) h->axis_ihl[d][i] = 2. / (a[i + 1] - a[i]);
  }
  return true;
}

// cell.tcc:335-384 for cell c on the host (host twin of cell_point_in)
bool host_point_in(mpm_gpu_t h, int64_t c, const double* p, double* xi) {
  const CellGeom& g = h->geom[c];
  if (h->isoparametric && !h->structured) {
    double X[8 * 3];
    for (int i = 0; i < h->nv; ++i)
      for (int d = 0; d < h->dim; ++d)
        X[i * h->dim + d] = h->coords[(size_t)h->cell_nodes[(size_t)c * h->nv + i] * h->dim + d];
    return h->dim == 2 ? point_in_cell_iso<2>(p, X, g.centroid, g.mean_length, xi)
                       : point_in_cell_iso<3>(p, X, g.centroid, g.mean_length, xi);
  }
  return h->dim == 2 ? point_in_cell<2>(p, g.centroid, g.len, g.mean_length, xi)
                     : point_in_cell<3>(p, g.centroid, g.len, g.mean_length, xi);
}

// first cell in id order containing p (host twin of the device fallback)
int32_t host_scan(mpm_gpu_t h, const double* p) {
  if (h->structured) {
    const double* ax[3] = {h->axis[0].data(), h->axis[1].data(), h->axis[2].data()};
    return h->dim == 2 ? structured_scan<2>(p, h->gcells, ax, h->geom.data())
                       : structured_scan<3>(p, h->gcells, ax, h->geom.data());
  }
  int64_t b[3] = {0, 0, 0};
  for (int i = 0; i < h->dim; ++i) {
    const double f = std::floor((p[i] - h->bmin[i]) / h->bsize[i]);
    if (!(f >= 0) || f >= (double)h->bn[i]) return -1;
    b[i] = (int64_t)f;
  }
  const int64_t bi = (b[2] * h->bn[1] + b[1]) * h->bn[0] + b[0];
  for (int32_t j = h->bin_off[bi]; j < h->bin_off[bi + 1]; ++j) {
    const int32_t c = h->bin_cells[j];
    double xi[3];
    if (host_point_in(h, c, p, xi)) return c;
  }
  return -1;
}

// MohrCoulomb / LinearElastic constructors (mohr_coulomb.tcc:3-81,
// linear_elastic.tcc:3-49) from the reference's JSON property object
MaterialParams make_material(int dim, const std::string& type, const Json& j) {
  MaterialParams m{};
  std::string base = type;
  const std::string suffix = dim == 2 ? "2D" : "3D";
  if (base.size() < 2 || base.substr(base.size() - 2) != suffix)
    throw InvalidArg("material type \"" + type + "\" does not match the " + suffix + " solver");
  base = base.substr(0, base.size() - 2);
  auto req = [&](const char* k) {
    if (!j.contains(k)) throw InvalidArg(std::string("material parameter not set: ") + k);
    return j.at(k).as_double();
  };
  m.density = req("density");
  m.E = req("youngs_modulus");
  m.nu = req("poisson_ratio");
  if (base == "LinearElastic") {
    if (j.contains("stress_rate") && j.at("stress_rate").is_string() &&
        (j.at("stress_rate").as_string() == "jaumann" ||
         j.at("stress_rate").as_string() == "green_naghdi"))
      throw InvalidArg("objective stress rates are not implemented on this path");
    m.type = 0;
    m.bulk = m.E / (3.0 * (1. - 2. * m.nu));
    m.shear = m.E / (2.0 * (1. + m.nu));
  } else if (base == "MohrCoulomb") {
    m.type = 1;
    double packing = 1.;
    if (j.contains("packing_fraction"))
      packing = j.at("packing_fraction").as_double();
    else if (j.contains("porosity"))
      packing = 1. - j.at("porosity").as_double();
    const bool wet = j.contains("porosity") &&
                     (j.contains("k_x") || j.contains("k_y") || j.contains("k_z"));
    m.grain_density = wet ? m.density : m.density / packing;
    m.min_packing = j.get("packing_fraction_minimum", 0.0);
    if (!j.contains("softening")) throw InvalidArg("material parameter not set: softening");
    m.softening = j.at("softening").as_bool() ? 1 : 0;
    m.phi_peak = req("friction") * kPiD / 180.;
    m.psi_peak = req("dilation") * kPiD / 180.;
    m.c_peak = req("cohesion");
    m.phi_res = req("residual_friction") * kPiD / 180.;
    m.psi_res = req("residual_dilation") * kPiD / 180.;
    m.c_res = req("residual_cohesion");
    m.pd_peak = req("peak_pdstrain");
    m.pd_res = req("residual_pdstrain");
    m.tension_cutoff = req("tension_cutoff");
    m.bulk = m.E / (3.0 * (1. - 2. * m.nu));
    m.shear = m.E / (2.0 * (1 + m.nu));
    const double apex = m.c_peak / std::tan(m.phi_peak);
    m.tc_init = check_low(m.tension_cutoff < apex ? m.tension_cutoff : apex);
    m.sin_phi = std::sin(m.phi_peak);
    m.cos_phi = std::cos(m.phi_peak);
    m.tan_phi = std::tan(m.phi_peak);
    m.tan_psi = std::tan(m.psi_peak);
  } else {
    throw InvalidArg("unknown material type \"" + type + "\"");
  }
  const double G = m.shear;
  m.a1 = m.bulk + (4.0 / 3.0) * G;
  m.a2 = m.bulk - (2.0 / 3.0) * G;
  return m;
}

void mc_init_state(const MaterialParams& m, double* sv) {
  sv[SV_YIELD] = 0;
  sv[SV_PHI] = m.phi_peak;
  sv[SV_PSI] = m.psi_peak;
  sv[SV_COH] = m.c_peak;
  sv[SV_TC] = m.tc_init;
  sv[SV_EPS] = sv[SV_RHO] = sv[SV_THETA] = sv[SV_PD] = 0.;
}

void upload_mesh(mpm_gpu_t h) {
  cudaStream_t st = h->stream;
  const int dim = h->dim;
  std::vector<double> nc((size_t)dim * h->nnodes);
  for (int64_t n = 0; n < h->nnodes; ++n)
    for (int d = 0; d < dim; ++d) nc[(size_t)d * h->nnodes + n] = h->coords[n * dim + d];
  h->d_ncoord.upload(nc.data(), nc.size(), st);
  h->d_cell_nodes.upload(h->cell_nodes.data(), h->cell_nodes.size(), st);
  h->d_geom.upload(h->geom.data(), h->geom.size(), st);
  h->d_nb_off.upload(h->nb_off.data(), h->nb_off.size(), st);
  h->d_nb.alloc(std::max<size_t>(1, h->nb.size()));
  h->d_nb.upload(h->nb.data(), h->nb.size(), st);
  h->d_bin_off.upload(h->bin_off.data(), h->bin_off.size(), st);
  h->d_bin_cells.alloc(std::max<size_t>(1, h->bin_cells.size()));
  h->d_bin_cells.upload(h->bin_cells.data(), h->bin_cells.size(), st);
  h->d_nf.alloc((size_t)h->nnf() * h->nnodes);
  h->d_active.alloc(h->nnodes);
  ck(cudaMemsetAsync(h->d_active.p, 0, h->nnodes, st), "memset");
  ck(cudaMemsetAsync(h->d_nf.p, 0, sizeof(double) * h->nnf() * h->nnodes, st), "memset");
  h->d_words.alloc(8);
  ck(cudaMemsetAsync(h->d_words.p, 0, sizeof(unsigned) * 8, st), "memset");
  if (h->structured)
    for (int d = 0; d < 3; ++d) {
      h->d_axis[d].upload(h->axis[d].data(), h->axis[d].size(), st);
      h->d_axis_ihl[d].upload(h->axis_ihl[d].data(), h->axis_ihl[d].size(), st);
    }
  if (h->mixed) {
    std::vector<float> f(h->dndx_c.begin(), h->dndx_c.end());
    h->d_dndx_cf.upload(f.data(), f.size(), st);
    h->d_nfv.alloc((size_t)nfv_stride(dim) * h->nnodes);
    ck(cudaMemsetAsync(h->d_nfv.p, 0, sizeof(float) * nfv_stride(dim) * h->nnodes, st), "memset");
    ck(cudaStreamSynchronize(st), "sync");  // f is a stack temporary
  } else {
    h->d_dndx_c.upload(h->dndx_c.data(), h->dndx_c.size(), st);
  }
  if (!h->structured) {
    h->d_nc_off.upload(h->nc_off.data(), h->nc_off.size(), st);
    h->d_nc_cell.alloc(std::max<size_t>(1, h->nc_cell.size()));
    h->d_nc_cell.upload(h->nc_cell.data(), h->nc_cell.size(), st);
    h->d_nc_slot.alloc(std::max<size_t>(1, h->nc_slot.size()));
    h->d_nc_slot.upload(h->nc_slot.data(), h->nc_slot.size(), st);
  }
  if (h->mixed)
    h->d_partials_f.alloc((size_t)h->ncells * h->nv * mixed_nval(dim));
  else
    h->d_partials.alloc((size_t)h->ncells * h->nv * (1 + 3 * dim));
  h->d_cnt.alloc(h->ncells);
  h->d_start.alloc(h->ncells + 1);
  const int64_t nb = (h->ncells + SCAN_BLOCK - 1) / SCAN_BLOCK;
  h->d_bsum.alloc(2 * nb + 2);
}

void upload_bcs(mpm_gpu_t h) {
  std::vector<int32_t> index(h->nnodes, -1);
  std::vector<NodeBC> table;
  std::map<std::string, int> dedup;
  for (auto& kv : h->bcs) {
    NodeBC b{};
    for (auto& c : kv.second.vel) {
      b.vel_mask |= (uint8_t)(1u << c.first);
      b.vel[c.first] = c.second;
    }
    for (auto& c : kv.second.acc) {
      b.acc_mask |= (uint8_t)(1u << c.first);
      b.acc[c.first] = c.second;
    }
    b.friction = kv.second.friction ? 1 : 0;
    b.fric_dir = (uint8_t)kv.second.fdir;
    b.fric_sign = kv.second.fsign;
    b.mu = kv.second.mu;
    if (kv.second.rotated) {
      b.rotated = 1;
      euler_rotation(h->dim, kv.second.angles, b.rot);
      // the inverse of the leading dim x dim block (Eigen's fixed-size inverse)
      double Rd[9], Ri[9];
      for (int a = 0; a < h->dim; ++a)
        for (int c = 0; c < h->dim; ++c) Rd[a * h->dim + c] = b.rot[a * 3 + c];
      if (h->dim == 2)
        inverse<2>(Rd, Ri);
      else
        inverse<3>(Rd, Ri);
      for (int a = 0; a < h->dim; ++a)
        for (int c = 0; c < h->dim; ++c) b.irot[a * 3 + c] = Ri[a * h->dim + c];
    }
    std::string key(reinterpret_cast<const char*>(&b), sizeof(b));
    auto it = dedup.find(key);
    int slot;
    if (it == dedup.end()) {
      slot = (int)table.size();
      table.push_back(b);
      dedup[key] = slot;
    } else {
      slot = it->second;
    }
    index[kv.first] = slot;
  }
  if (table.empty()) table.push_back(NodeBC{});
  h->d_bcs.upload(table.data(), table.size(), h->stream);
  h->d_bc_index.upload(index.data(), index.size(), h->stream);
}

void upload_pvc(mpm_gpu_t h) {
  std::vector<int16_t> idx(h->npad, -1);
  std::vector<ParticleVC> table;
  std::map<std::string, int> dedup;
  for (const auto& pc : h->p_vc) {
    const int64_t p = pc.first;
    if (p >= h->np || pc.second.empty()) continue;
    ParticleVC r{};
    for (auto& c : pc.second) {
      r.mask |= 1u << c.first;
      r.value[c.first] = c.second;
    }
    std::string key(reinterpret_cast<const char*>(&r), sizeof(r));
    auto it = dedup.find(key);
    int slot;
    if (it == dedup.end()) {
      slot = (int)table.size();
      if (slot > 32767) throw InvalidArg("too many distinct particle velocity constraints");
      table.push_back(r);
      dedup[key] = slot;
    } else {
      slot = it->second;
    }
    idx[p] = (int16_t)slot;
  }
  if (table.empty()) table.push_back(ParticleVC{});
  h->d_pvcs.upload(table.data(), table.size(), h->stream);
  h->d_pvc.upload(idx.data(), idx.size(), h->stream);
  h->p_vc_dirty = false;
}

// Particle buffers for h->npad rows; a buffer that already has its size (a
// state of the same particle count loaded again) is kept.
void allocate_particles(mpm_gpu_t h) {
  const int64_t np = h->npad;
  h->d_pf.resize((size_t)(h->mixed ? h->nfields_x() : h->nfields()) * np);
  if (h->mixed) h->d_pm.resize((size_t)h->nfields_m() * np);
  h->d_cell.resize(np);
  h->d_mat.resize(np);
  if (h->cfg.scheme == MPM_SCHEME_MUSL) h->d_xnext.resize((size_t)h->dim * np);
  if (h->cfg.velocity_update >= MPM_VELOCITY_ASFLIP) {
    h->d_mapb.resize((size_t)h->dim * h->dim * np);
    ck(cudaMemsetAsync(h->d_mapb.p, 0, sizeof(double) * h->dim * h->dim * np, h->stream),
       "memset");
  }
  h->d_lost.resize(std::max<int64_t>(1, np));
  h->d_rank.resize(std::max<int64_t>(1, np));
  h->d_order.resize(std::max<int64_t>(1, np));
  h->any_mc = false;
  for (auto& m : h->mats) h->any_mc = h->any_mc || m.type == 1;
  if (h->any_mc) {
    h->d_plist.resize(np);
    h->d_pbuf.resize((size_t)7 * np);
    h->d_rpass.resize(std::max<int64_t>(1, np));
    ck(cudaMemsetAsync(h->d_rpass.p, 0, std::max<int64_t>(1, np), h->stream), "memset");
  } else {
    h->d_plist.free();
    h->d_pbuf.free();
    h->d_rpass.free();
  }
  if (h->any_mc && h->mixed)
    h->d_svf.resize((size_t)SVF_N * np);
  else
    h->d_svf.free();
  if (h->any_mc && !h->mixed)
    h->d_sv.resize((size_t)SV_N * np);
  else
    h->d_sv.free();
}

void refresh_state(mpm_gpu_t h) {
  DevState& s = h->ds;
  s.np = h->npad;
  s.pf = h->d_pf.p;
  s.sv = h->d_sv.p;
  s.mapb = h->d_mapb.p;
  s.iso = h->isoparametric && !h->structured ? 1 : 0;
  s.cell = h->d_cell.p;
  s.mat = h->d_mat.p;
  s.pvc = h->d_pvc.p;
  s.nn = h->nnodes;
  s.nf = h->d_nf.p;
  s.active = h->d_active.p;
  s.bc_index = h->d_bc_index.p;
  s.ncells = h->ncells;
  s.cell_nodes = h->d_cell_nodes.p;
  s.ncoord = h->d_ncoord.p;
  s.geom = h->d_geom.p;
  s.nb_off = h->d_nb_off.p;
  s.nb = h->d_nb.p;
  s.bin_off = h->d_bin_off.p;
  s.bin_cells = h->d_bin_cells.p;
  for (int i = 0; i < 3; ++i) {
    s.bmin[i] = h->bmin[i];
    s.bsize[i] = h->bsize[i];
    s.bn[i] = h->bn[i];
  }
  s.structured = h->structured ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    s.gcells[d] = h->gcells[d];
    s.axis[d] = h->d_axis[d].p;
    s.axis_ihl[d] = h->d_axis_ihl[d].p;
  }
  s.nc_off = h->d_nc_off.p;
  s.nc_cell = h->d_nc_cell.p;
  s.nc_slot = h->d_nc_slot.p;
  s.dndx_c = h->d_dndx_c.p;
  s.cnt = h->d_cnt.p;
  s.start = h->d_start.p;
  s.rank = h->d_rank.p;
  s.order = h->d_order.p;
  s.bsum = h->d_bsum.p;
  s.partials = h->d_partials.p;
  s.lost = h->d_lost.p;
  s.xnext = h->d_xnext.p;
  s.nlost = h->d_words.p;
  s.err = h->d_words.p + 1;
  s.nplastic = h->d_words.p + 2;
  s.nplastic_heavy = h->d_words.p + 3;
  for (int k = 0; k < MAX_TANGENTS; ++k) {
    const bool on = h->ntangent > 0;
    s.pft[k] = on ? h->d_pft[k].p : nullptr;
    s.svt[k] = on ? h->d_svt[k].p : nullptr;
    s.nft[k] = on ? h->d_nft[k].p : nullptr;
    s.partt[k] = on ? h->d_partt[k].p : nullptr;
  }
  s.mats_t = h->ntangent > 0 ? h->d_mats_t.p : nullptr;
  s.tpbuf = h->ntangent > 0 ? h->d_tpbuf.p : nullptr;
  s.tangent_mass_floor = h->tangent_mass_floor;
  s.any_softening = 0;
  for (auto& m : h->mats) s.any_softening |= (m.type == 1 && m.softening) ? 1 : 0;
  s.plist = h->any_mc ? h->d_plist.p : nullptr;
  s.rpass = h->any_mc ? h->d_rpass.p : nullptr;
  s.pbuf = h->any_mc ? h->d_pbuf.p : nullptr;
  s.pbuf_f = h->any_mc ? reinterpret_cast<float*>(h->d_pbuf.p) : nullptr;
  s.mats = h->d_mats.p;
  s.bcs = h->d_bcs.p;
  s.pvcs = h->d_pvcs.p;
  s.pm = h->d_pm.p;
  s.svf = h->d_svf.p;
  s.nfv = h->d_nfv.p;
  s.partials_f = h->d_partials_f.p;
  s.dndx_cf = h->d_dndx_cf.p;
  s.mats_f = h->d_mats_f.p;
}

// Offsets of the FP64 particle layout (PF) for the solver's dimension.
struct Layout {
  int X, U, V, S, E, F, VOL, RHO, MASS, NF, NS, NE, NFG;
};
Layout layout(int dim) {
  if (dim == 2)
    return {PF<2>::X, PF<2>::U,   PF<2>::V,    PF<2>::S,  PF<2>::E,  PF<2>::F,  PF<2>::VOL,
            PF<2>::RHO, PF<2>::MASS, PF<2>::NF, PF<2>::NS, PF<2>::NE, PF<2>::NFG};
  return {PF<3>::X, PF<3>::U,   PF<3>::V,    PF<3>::S,  PF<3>::E,  PF<3>::F,  PF<3>::VOL,
          PF<3>::RHO, PF<3>::MASS, PF<3>::NF, PF<3>::NS, PF<3>::NE, PF<3>::NFG};
}
struct LayoutM {
  int V, S, E, H, V0, RHO0, JP, MASS, NF, PDS;
};
LayoutM layout_m(int dim) {
  if (dim == 2)
    return {PM<2>::V, PM<2>::S, PM<2>::E, PM<2>::H, PM<2>::V0, PM<2>::RHO0, PM<2>::JP, PM<2>::MASS,
            PM<2>::NF, PDX<2>::PDS};
  return {PM<3>::V, PM<3>::S, PM<3>::E, PM<3>::H, PM<3>::V0, PM<3>::RHO0, PM<3>::JP, PM<3>::MASS,
          PM<3>::NF, PDX<3>::PDS};
}
bool identity_entry(int dim, int k) { return dim == 2 ? (k == 0 || k == 3) : (k % 4 == 0); }

// Upload particle fields given in the FP64 layout (pf: [PF::NF][npad], sv:
// [SV_N][npad] or empty).  The mixed path keeps x, u and pdstrain in FP64 and
// stores the rest in FP32, F as H = F - I and volume / density as the initial
// values with P = V / V0 - 1 = 0.
void upload_particle_fields(mpm_gpu_t h, const std::vector<double>& pf, const std::vector<double>& sv) {
  const int64_t np = h->npad;
  const int dim = h->dim;
  if (!h->mixed) {
    h->d_pf.upload(pf.data(), pf.size(), h->stream);
    if (h->any_mc) h->d_sv.upload(sv.data(), sv.size(), h->stream);
    ck(cudaStreamSynchronize(h->stream), "sync");
    return;
  }
  const Layout L = layout(dim);
  const LayoutM M = layout_m(dim);
  std::vector<double> px((size_t)h->nfields_x() * np, 0.0);
  std::vector<float> pm((size_t)h->nfields_m() * np, 0.f);
  parallel_for(np, [&](int64_t pa, int64_t pb) {
  for (int64_t p = pa; p < pb; ++p) {
    auto f = [&](int o) { return pf[(size_t)o * np + p]; };
    for (int d = 0; d < dim; ++d) {
      px[(size_t)(PDX<3>::X + d) * np + p] = f(L.X + d);
      px[(size_t)(dim + d) * np + p] = f(L.U + d);
      pm[(size_t)(M.V + d) * np + p] = (float)f(L.V + d);
    }
    px[(size_t)M.PDS * np + p] = h->any_mc ? sv[(size_t)SV_PD * np + p] : 0.;
    for (int k = 0; k < L.NS; ++k) pm[(size_t)(M.S + k) * np + p] = (float)f(L.S + k);
    for (int k = 0; k < L.NE; ++k) pm[(size_t)(M.E + k) * np + p] = (float)f(L.E + k);
    for (int k = 0; k < L.NFG; ++k)
      pm[(size_t)(M.H + k) * np + p] = (float)(f(L.F + k) - (identity_entry(dim, k) ? 1. : 0.));
    pm[(size_t)M.V0 * np + p] = (float)f(L.VOL);
    pm[(size_t)M.RHO0 * np + p] = (float)f(L.RHO);
    pm[(size_t)M.JP * np + p] = 0.f;
    pm[(size_t)M.MASS * np + p] = (float)f(L.MASS);
  }
  });
  h->d_pf.upload(px.data(), px.size(), h->stream);
  h->d_pm.upload(pm.data(), pm.size(), h->stream);
  std::vector<float> svf;
  if (h->any_mc) {
    svf.resize((size_t)SVF_N * np);
    parallel_for((int64_t)svf.size(), [&](int64_t a, int64_t b) {
      for (int64_t i = a; i < b; ++i) svf[i] = (float)sv[i];
    });
    h->d_svf.upload(svf.data(), svf.size(), h->stream);
  }
  ck(cudaStreamSynchronize(h->stream), "sync");
}

// Pack host particle rows (ABI layout) into the device SoA field order.
void pack_particles(mpm_gpu_t h, const mpm_gpu_particles* in, const std::vector<int32_t>* cells) {
  const int dim = h->dim;
  const int64_t np = h->np, ns = h->npad;
  std::vector<double> pf((size_t)h->nfields() * ns, 0.0);
  auto at = [&](int f, int64_t p) -> double& { return pf[(size_t)f * ns + p]; };
  const int X = dim == 2 ? PF<2>::X : PF<3>::X, U = dim == 2 ? PF<2>::U : PF<3>::U;
  const int V = dim == 2 ? PF<2>::V : PF<3>::V, S = dim == 2 ? PF<2>::S : PF<3>::S;
  const int E = dim == 2 ? PF<2>::E : PF<3>::E, Fo = dim == 2 ? PF<2>::F : PF<3>::F;
  const int VOL = dim == 2 ? PF<2>::VOL : PF<3>::VOL, RHO = dim == 2 ? PF<2>::RHO : PF<3>::RHO;
  const int MASS = dim == 2 ? PF<2>::MASS : PF<3>::MASS;
  parallel_for(np, [&](int64_t pa, int64_t pb) {
  for (int64_t p = pa; p < pb; ++p) {
    for (int d = 0; d < dim; ++d) {
      at(X + d, p) = in->x ? in->x[p * 3 + d] : h->p_coords[p * dim + d];
      at(U + d, p) = in->u ? in->u[p * 3 + d] : 0.;
      at(V + d, p) = in->v ? in->v[p * 3 + d] : 0.;
    }
    if (dim == 2) {
      const int smap[4] = {0, 1, 2, 3};
      for (int k = 0; k < 4; ++k) at(S + k, p) = in->stress ? in->stress[p * 6 + smap[k]] : 0.;
      if (in->stress && (in->stress[p * 6 + 4] != 0. || in->stress[p * 6 + 5] != 0.))
        throw InvalidArg("2D particle stress must have zero yz and xz components");
      const int emap[3] = {0, 1, 3};
      for (int k = 0; k < 3; ++k) at(E + k, p) = in->strain ? in->strain[p * 6 + emap[k]] : 0.;
      if (in->strain && (in->strain[p * 6 + 2] != 0. || in->strain[p * 6 + 4] != 0. ||
                         in->strain[p * 6 + 5] != 0.))
        throw InvalidArg("2D particle strain must have zero zz, yz and xz components");
      const int fmap[4] = {0, 1, 3, 4};
      for (int k = 0; k < 4; ++k) at(Fo + k, p) = in->F ? in->F[p * 9 + fmap[k]] : (k == 0 || k == 3 ? 1. : 0.);
      if (in->F && (in->F[p * 9 + 2] != 0. || in->F[p * 9 + 5] != 0. || in->F[p * 9 + 6] != 0. ||
                    in->F[p * 9 + 7] != 0. || in->F[p * 9 + 8] != 1.))
        throw InvalidArg("2D deformation gradient must have third row and column (0,0,1)");
    } else {
      for (int k = 0; k < 6; ++k) {
        at(S + k, p) = in->stress ? in->stress[p * 6 + k] : 0.;
        at(E + k, p) = in->strain ? in->strain[p * 6 + k] : 0.;
      }
      for (int k = 0; k < 9; ++k) at(Fo + k, p) = in->F ? in->F[p * 9 + k] : (k % 4 == 0 ? 1. : 0.);
    }
    const MaterialParams& m = h->mats[h->p_mat[p]];
    at(RHO, p) = in->density ? in->density[p] : m.density;
    at(VOL, p) = in->volume ? in->volume[p] : 0.;
    at(MASS, p) = in->mass ? in->mass[p] : at(VOL, p) * at(RHO, p);
  }
  });
  std::vector<int32_t> cell(ns, -1);
  parallel_for(np, [&](int64_t pa, int64_t pb) {
  for (int64_t p = pa; p < pb; ++p) {
    if (in->cell) {
      const int64_t c = in->cell[p];
      if (c < -1 || c >= h->ncells) throw InvalidArg("particle cell id out of range");
      cell[p] = (int32_t)c;
    } else {
      cell[p] = (*cells)[p];
    }
  }
  });
  h->d_cell.upload(cell.data(), ns, h->stream);
  std::vector<uint16_t> mat(h->p_mat);
  mat.resize(ns, 0);
  h->d_mat.upload(mat.data(), ns, h->stream);
  std::vector<double> sv;
  if (h->any_mc) {
    sv.assign((size_t)SV_N * ns, 0.0);
    parallel_for(np, [&](int64_t pa, int64_t pb) {
    for (int64_t p = pa; p < pb; ++p) {
      const MaterialParams& m = h->mats[h->p_mat[p]];
      double s[SV_N] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      if (in->svars)
        for (int k = 0; k < SV_N; ++k) s[k] = in->svars[p * SV_N + k];
      else if (m.type == 1)
        mc_init_state(m, s);
      for (int k = 0; k < SV_N; ++k) sv[(size_t)k * ns + p] = s[k];
    }
    });
  }
  upload_particle_fields(h, pf, sv);
  ck(cudaStreamSynchronize(h->stream), "sync");
}

// The caller's particle arrays (rows as in mpm_gpu_particles) placed one after
// another in h->d_rows; an array whose pointer is null gets offset -1.
template <class P>
RowStage stage_rows(mpm_gpu_t h, int64_t n, P* const (&ptr)[10], int64_t& total) {
  static constexpr int width[10] = {3, 3, 3, 6, 6, 9, 1, 1, 1, SV_N};
  int64_t off[10];
  total = 0;
  for (int k = 0; k < 10; ++k) {
    off[k] = ptr[k] ? total : -1;
    if (ptr[k]) total += (int64_t)width[k] * n;
  }
  if ((size_t)total > h->d_rows.n) h->d_rows.alloc((size_t)total);
  RowStage r{n, h->d_rows.p, off[0], off[1], off[2], off[3], off[4], off[5], off[6], off[7], off[8], off[9]};
  return r;
}
int row_width(int k) {
  static constexpr int width[10] = {3, 3, 3, 6, 6, 9, 1, 1, 1, SV_N};
  return width[k];
}

// A pinned host buffer of at least n doubles for the staged rows (two chunks),
// kept by the handle; null when the host cannot pin that much (the copies then
// go to and from the caller's pageable arrays directly).
double* pinned_rows(mpm_gpu_t h, int64_t n) {
  if ((size_t)n <= h->h_rows_n) return h->h_rows;
  if (h->h_rows) cudaFreeHost(h->h_rows);
  h->h_rows = nullptr;
  h->h_rows_n = 0;
  if (cudaHostAlloc(reinterpret_cast<void**>(&h->h_rows), sizeof(double) * n, cudaHostAllocDefault) !=
      cudaSuccess) {
    cudaGetLastError();  // clear the failed allocation's error
    h->h_rows = nullptr;
    return nullptr;
  }
  h->h_rows_n = (size_t)n;
  return h->h_rows;
}

// dst[0, n) = src[0, n) on all host threads
void parallel_copy(double* dst, const double* src, int64_t n) {
  parallel_for(n, [&](int64_t a, int64_t b) { std::memcpy(dst + a, src + a, sizeof(double) * (b - a)); });
}

// Staged rows move through pinned memory in chunks of ROW_CHUNK doubles (64 MiB),
// two in flight: the host gathers (or scatters) one chunk on all its threads
// while the DMA engine copies the other.
constexpr int64_t ROW_CHUNK = (int64_t)8 << 20;

// The part [lo, hi) of the staged-row index space (the arrays one after another
// at their offsets) copied between the caller's arrays and buf, which holds
// index lo at buf[0].
template <class P>
void rows_range(P* const (&ptr)[10], const int64_t (&off)[10], int64_t np, int64_t lo, int64_t hi,
                double* buf, bool gather) {
  for (int k = 0; k < 10; ++k) {
    if (!ptr[k]) continue;
    const int64_t a = off[k], b = a + (int64_t)row_width(k) * np;
    const int64_t s0 = std::max(a, lo), s1 = std::min(b, hi);
    if (s0 >= s1) continue;
    if (gather)
      parallel_copy(buf + (s0 - lo), ptr[k] + (s0 - a), s1 - s0);
    else if constexpr (!std::is_const<P>::value)
      parallel_copy(ptr[k] + (s0 - a), buf + (s0 - lo), s1 - s0);
  }
}

// True when each given array lies in page-locked host memory (its first and
// last byte), so the DMA engine can copy it without staging.
template <class P>
bool page_locked(P* const (&ptr)[10], int64_t np) {
  bool any = false;
  for (int k = 0; k < 10; ++k) {
    if (!ptr[k] || np == 0) continue;
    const char* a = reinterpret_cast<const char*>(ptr[k]);
    for (const char* q : {a, a + sizeof(double) * row_width(k) * np - 1}) {
      cudaPointerAttributes attr{};
      if (cudaPointerGetAttributes(&attr, q) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      if (attr.type != cudaMemoryTypeHost) return false;
    }
    any = true;
  }
  return any;
}

void ensure_stage_events(mpm_gpu_t h) {
  for (auto& e : h->stage_ev)
    if (!e) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
}

// Load a full particle state (every field given) with plain copies into the
// staging buffer and one device kernel that writes the device layout, the
// same values pack_particles writes.  Cell ids, material slots and the 2D
// zero-component checks stay on the host.
void load_rows_device(mpm_gpu_t h, const mpm_gpu_particles* in) {
  const int dim = h->dim;
  const int64_t np = h->np, ns = h->npad;
  if (dim == 2)
    parallel_for(np, [&](int64_t pa, int64_t pb) {
      for (int64_t p = pa; p < pb; ++p) {
        const double *sg = in->stress + p * 6, *ep = in->strain + p * 6, *F = in->F + p * 9;
        if (sg[4] != 0. || sg[5] != 0.)
          throw InvalidArg("2D particle stress must have zero yz and xz components");
        if (ep[2] != 0. || ep[4] != 0. || ep[5] != 0.)
          throw InvalidArg("2D particle strain must have zero zz, yz and xz components");
        if (F[2] != 0. || F[5] != 0. || F[6] != 0. || F[7] != 0. || F[8] != 1.)
          throw InvalidArg("2D deformation gradient must have third row and column (0,0,1)");
      }
    });
  std::vector<int32_t> cell(ns, -1);
  parallel_for(np, [&](int64_t pa, int64_t pb) {
    for (int64_t p = pa; p < pb; ++p) {
      const int64_t c = in->cell[p];
      if (c < -1 || c >= h->ncells) throw InvalidArg("particle cell id out of range");
      cell[p] = (int32_t)c;
    }
  });
  h->d_cell.upload(cell.data(), ns, h->stream);
  std::vector<uint16_t> mat(h->p_mat);
  mat.resize(ns, 0);
  h->d_mat.upload(mat.data(), ns, h->stream);
  const double* const ptr[10] = {in->x, in->u, in->v, in->stress, in->strain, in->F,
                                 in->volume, in->mass, in->density, h->any_mc ? in->svars : nullptr};
  int64_t total = 0;
  const RowStage r = stage_rows(h, np, ptr, total);
  const int64_t off[10] = {r.x, r.u, r.v, r.stress, r.strain, r.F, r.volume, r.mass, r.density, r.svars};
  const int64_t chunk = std::min(total, ROW_CHUNK);
  const bool direct = page_locked(ptr, np);
  if (direct) {
    for (int k = 0; k < 10; ++k)
      if (ptr[k] && np)
        ck(cudaMemcpyAsync(r.base + off[k], ptr[k], sizeof(double) * row_width(k) * np,
                           cudaMemcpyHostToDevice, h->stream), "H2D");
  } else if (double* pin = total ? pinned_rows(h, 2 * chunk) : nullptr) {
    ensure_stage_events(h);
    bool busy[2] = {false, false};
    int k = 0;
    for (int64_t lo = 0; lo < total; lo += chunk, k ^= 1) {
      const int64_t hi = std::min(total, lo + chunk);
      if (busy[k]) ck(cudaEventSynchronize(h->stage_ev[k]), "row copy");
      rows_range(ptr, off, np, lo, hi, pin + k * chunk, true);
      ck(cudaMemcpyAsync(r.base + lo, pin + k * chunk, sizeof(double) * (hi - lo),
                         cudaMemcpyHostToDevice, h->stream), "H2D");
      ck(cudaEventRecord(h->stage_ev[k], h->stream), "cudaEventRecord");
      busy[k] = true;
    }
  } else {
    for (int k = 0; k < 10; ++k)
      if (ptr[k] && np)
        ck(cudaMemcpyAsync(r.base + off[k], ptr[k], sizeof(double) * row_width(k) * np,
                           cudaMemcpyHostToDevice, h->stream), "H2D");
  }
  refresh_state(h);
  launch_rows_to_state(dim, h->mixed, h->any_mc, h->ds, r, h->stream);
  ck(cudaGetLastError(), "rows to state");
  ck(cudaStreamSynchronize(h->stream), "sync");
}

#define MPM_GUARD(h)                                                   \
  if (!(h)) return MPM_ERR_INVALID;                                    \
  try {
#define MPM_END(h)                                                     \
  }                                                                    \
  catch (const InvalidArg& e) { return fail(h, MPM_ERR_INVALID, e.what()); } \
  catch (const CudaError& e) { return fail(h, MPM_ERR_CUDA, e.what()); }     \
  catch (const std::exception& e) { return fail(h, MPM_ERR_INVALID, e.what()); }

}  // namespace

namespace mpm_b200 {
// the material factory of the C ABI, shared with the no-allocation entry point
MaterialParams material_from_json(int dim, const char* type, const char* json_props) {
  return make_material(dim, type, parse_json(json_props));
}
}  // namespace mpm_b200

extern "C" {

const char* mpm_gpu_version(void) { return MPM_VERSION; }

int mpm_gpu_host_alloc(size_t bytes, void** ptr) {
  if (!ptr) return MPM_ERR_INVALID;
  *ptr = nullptr;
  if (cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocPortable) != cudaSuccess) {  // every device's context
    cudaGetLastError();
    *ptr = nullptr;
    return MPM_ERR_ALLOC;
  }
  return MPM_OK;
}

int mpm_gpu_host_free(void* ptr) {
  if (ptr && cudaFreeHost(ptr) != cudaSuccess) {
    cudaGetLastError();
    return MPM_ERR_CUDA;
  }
  return MPM_OK;
}

int mpm_gpu_create(const mpm_gpu_config* cfg, mpm_gpu_t* out) {
  if (!cfg || !out) return MPM_ERR_INVALID;
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return MPM_ERR_INVALID;
  if (cfg->scheme != MPM_SCHEME_USF && cfg->scheme != MPM_SCHEME_USL &&
      cfg->scheme != MPM_SCHEME_MUSL)
    return MPM_ERR_UNSUPPORTED;
  if (cfg->velocity_update < MPM_VELOCITY_FLIP || cfg->velocity_update > MPM_VELOCITY_APIC)
    return MPM_ERR_UNSUPPORTED;
  // the mapping-matrix updates run on the USF / USL paths (MUSL's second
  // mapping would take its branch vectors from the updated positions)
  if (cfg->velocity_update >= MPM_VELOCITY_ASFLIP && cfg->scheme == MPM_SCHEME_MUSL)
    return MPM_ERR_UNSUPPORTED;
  if (cfg->precision != MPM_PRECISION_FP64 && cfg->precision != MPM_PRECISION_MIXED)
    return MPM_ERR_UNSUPPORTED;
  if (!(cfg->dt > 0)) return MPM_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MPM_ERR_CUDA;
  if (cfg->device < 0 || cfg->device >= ndev) return MPM_ERR_INVALID;
  auto* h = new mpm_gpu_solver();
  h->cfg = *cfg;
  h->dim = cfg->dim;
  h->nv = cfg->dim == 2 ? 4 : 8;
  h->mixed = cfg->precision == MPM_PRECISION_MIXED;
  // test hook (MPM_B200_TEST_WAIT_TIMEOUT=1): the staged G2P's first copy wait
  // runs out on purpose, so the MPM_ERR_TIMEOUT path can be exercised
  if (const char* e = std::getenv("MPM_B200_TEST_WAIT_TIMEOUT")) h->ds.test_wait_timeout = std::atoi(e) != 0;
  if (cudaSetDevice(cfg->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return MPM_ERR_CUDA;
  }
  *out = h;
  return MPM_OK;
}

int mpm_gpu_destroy(mpm_gpu_t h) {
  if (!h) return MPM_ERR_INVALID;
  cudaSetDevice(h->cfg.device);
  if (h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  if (h->h_stage) cudaFreeHost(h->h_stage);
  if (h->h_rows) cudaFreeHost(h->h_rows);
  for (auto& e : h->stage_ev)
    if (e) cudaEventDestroy(e);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->pgraph) cudaGraphExecDestroy(h->pgraph);
  delete h;
  return MPM_OK;
}

const char* mpm_gpu_last_error(mpm_gpu_t h) { return h ? h->err.c_str() : "null handle"; }

int mpm_gpu_set_mesh(mpm_gpu_t h, int64_t nnodes, const double* coords, int64_t ncells,
                     int32_t npc, const int64_t* cell_nodes) {
  MPM_GUARD(h)
  if (npc != h->nv) throw InvalidArg("nodes_per_cell must be 4 (2D quad4) or 8 (3D hex8)");
  if (nnodes <= 0 || ncells <= 0 || !coords || !cell_nodes) throw InvalidArg("empty mesh");
  if (nnodes > INT32_MAX || ncells > INT32_MAX / 8) throw InvalidArg("mesh too large for 32-bit indices");
  if (ncells > (int64_t)SCAN_BLOCK * SCAN_BLOCK) throw InvalidArg("mesh too large for the cell sort");
  if (h->mesh_set) throw InvalidArg("mesh already set");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int dim = h->dim, nv = h->nv;
  h->nnodes = nnodes;
  h->ncells = ncells;
  h->coords.assign(coords, coords + nnodes * dim);
  h->cell_nodes.resize((size_t)ncells * nv);
  h->geom.resize(ncells);
  h->cell_volume.resize(ncells);
  std::vector<double> X(nv * dim);
  for (int64_t c = 0; c < ncells; ++c) {
    for (int i = 0; i < nv; ++i) {
      const int64_t n = cell_nodes[c * nv + i];
      if (n < 0 || n >= nnodes) throw InvalidArg("cell node id out of range");
      h->cell_nodes[c * nv + i] = (int32_t)n;
      for (int d = 0; d < dim; ++d) X[i * dim + d] = coords[n * dim + d];
    }
    cell_geometry(dim, X.data(), &h->geom[c], &h->cell_volume[c]);
    if (!(h->cell_volume[c] > 0)) throw InvalidArg("Negative or zero volume cell, misconfigured cell!");
  }
  // dN/dx at the cell centroid (cell.tcc:33-65), once per cell
  h->dndx_c.resize((size_t)ncells * nv * dim);
  for (int64_t c = 0; c < ncells; ++c) {
    for (int i = 0; i < nv; ++i) {
      const int64_t n = cell_nodes[c * nv + i];
      for (int d = 0; d < dim; ++d) X[i * dim + d] = coords[n * dim + d];
    }
    double xi0[3] = {0., 0., 0.};
    if (dim == 2)
      dn_dx<2>(xi0, X.data(), &h->dndx_c[(size_t)c * nv * dim]);
    else
      dn_dx<3>(xi0, X.data(), &h->dndx_c[(size_t)c * nv * dim]);
  }
  // A tensor-product grid needs no connectivity tables: node ids, neighbours
  // and the cells around a node follow from (i, j, k).
  h->structured = detect_structured(h);
  if (h->structured) {
    h->nc_off.assign(nnodes + 1, 0);
    h->nc_cell.clear();
    h->nc_slot.clear();
    h->nb_off.assign(ncells + 1, 0);
    h->nb.clear();
    h->bin_off.assign(2, 0);
    h->bin_cells.clear();
    upload_mesh(h);
    upload_bcs(h);  // every node gets a (possibly empty) constraint slot
    h->mesh_set = true;
    return MPM_OK;
  }
  std::vector<std::vector<int32_t>> node_cells(nnodes);
  for (int64_t c = 0; c < ncells; ++c)
    for (int i = 0; i < nv; ++i) node_cells[h->cell_nodes[c * nv + i]].push_back((int32_t)c);
  // node -> (cell, slot), ascending cell id, for the nodal gather on general meshes
  h->nc_off.assign(nnodes + 1, 0);
  for (int64_t n = 0; n < nnodes; ++n) h->nc_off[n + 1] = h->nc_off[n] + (int32_t)node_cells[n].size();
  h->nc_cell.resize(h->nc_off[nnodes]);
  h->nc_slot.resize(h->nc_off[nnodes]);
  for (int64_t n = 0; n < nnodes; ++n) {
    std::vector<int32_t> cs = node_cells[n];
    std::sort(cs.begin(), cs.end());
    cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
    int32_t e = h->nc_off[n];
    for (int32_t c : cs) {
      for (int i = 0; i < nv; ++i)
        if (h->cell_nodes[(size_t)c * nv + i] == n) {
          h->nc_cell[e] = c;
          h->nc_slot[e] = (int8_t)i;
          ++e;
          break;
        }
    }
    h->nc_off[n + 1] = e;  // duplicates (a node listed twice in a cell) counted once
  }
  // mesh.tcc:287-306 neighbours: cells sharing a node, ascending id
  h->nb_off.assign(ncells + 1, 0);
  h->nb.clear();
  std::vector<int32_t> tmp;
  for (int64_t c = 0; c < ncells; ++c) {
    tmp.clear();
    for (int i = 0; i < nv; ++i)
      for (int32_t o : node_cells[h->cell_nodes[c * nv + i]])
        if (o != c) tmp.push_back(o);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    h->nb.insert(h->nb.end(), tmp.begin(), tmp.end());
    h->nb_off[c + 1] = (int32_t)h->nb.size();
  }
  build_bins(h);
  upload_mesh(h);
  upload_bcs(h);  // every node gets a (possibly empty) constraint slot
  h->mesh_set = true;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_add_material(mpm_gpu_t h, int32_t id, const char* type, const char* json_props) {
  MPM_GUARD(h)
  if (!type || !json_props) throw InvalidArg("null material type or properties");
  if (h->mat_index.count(id)) throw InvalidArg("New material cannot be added, insertion failed");
  if (h->mats.size() >= 65535) throw InvalidArg("too many materials");
  const Json j = parse_json(json_props);
  MaterialParams m = make_material(h->dim, type, j);
  h->mat_index[id] = (int)h->mats.size();
  h->mats.push_back(m);
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  h->d_mats.upload(h->mats.data(), h->mats.size(), h->stream);
  if (h->mixed) {
    std::vector<MaterialT<float>> mf;
    for (auto& x : h->mats) mf.push_back(material_cast<float>(x));
    h->d_mats_f.upload(mf.data(), mf.size(), h->stream);
  }
  ck(cudaStreamSynchronize(h->stream), "sync");
  MPM_END(h)
  return MPM_OK;
}

static int add_vel_acc(mpm_gpu_t h, int64_t n, const int64_t* nid, const int32_t* dir,
                       const double* val, bool vel) {
  MPM_GUARD(h)
  if (!h->mesh_set) throw InvalidArg("set the mesh first");
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= h->nnodes) throw InvalidArg("constraint node id out of range");
    if (dir[i] < 0 || dir[i] >= h->dim) throw InvalidArg("Constraint direction is out of bounds");
    HostBC& b = h->bcs[nid[i]];
    if (vel)
      b.vel.insert(std::make_pair((unsigned)dir[i], val[i]));
    else {
      if (b.vel.count((unsigned)dir[i]))
        throw InvalidArg("Acceleration and velocity constraints set in the same direction for the same node");
      b.acc.insert(std::make_pair((unsigned)dir[i], val[i]));
    }
  }
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  upload_bcs(h);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_add_velocity_constraints(mpm_gpu_t h, int64_t n, const int64_t* nid, const int32_t* dir,
                                     const double* val) {
  return add_vel_acc(h, n, nid, dir, val, true);
}

int mpm_gpu_add_acceleration_constraints(mpm_gpu_t h, int64_t n, const int64_t* nid,
                                         const int32_t* dir, const double* val) {
  return add_vel_acc(h, n, nid, dir, val, false);
}

int mpm_gpu_set_nodal_euler_angles(mpm_gpu_t h, int64_t n, const int64_t* nid,
                                   const double* angles) {
  MPM_GUARD(h)
  if (!h->mesh_set) throw InvalidArg("set the mesh first");
  if (n > 0 && (!nid || !angles)) throw InvalidArg("null node ids or angles");
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= h->nnodes) throw InvalidArg("Euler angle node id out of range");
    HostBC& b = h->bcs[nid[i]];
    b.rotated = true;
    for (int d = 0; d < 3; ++d) b.angles[d] = d < h->dim ? angles[i * h->dim + d] : 0.;
  }
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  upload_bcs(h);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_add_friction_constraints(mpm_gpu_t h, int64_t n, const int64_t* nid, const int32_t* dir,
                                     const int32_t* sign, const double* mu) {
  MPM_GUARD(h)
  if (!h->mesh_set) throw InvalidArg("set the mesh first");
  for (int64_t i = 0; i < n; ++i) {
    if (nid[i] < 0 || nid[i] >= h->nnodes) throw InvalidArg("constraint node id out of range");
    if (dir[i] < 0 || dir[i] >= h->dim) throw InvalidArg("Constraint direction is out of bounds");
    HostBC& b = h->bcs[nid[i]];
    b.friction = true;
    b.fdir = (unsigned)dir[i];
    b.fsign = sign[i];
    b.mu = mu[i];
  }
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  upload_bcs(h);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_add_particles(mpm_gpu_t h, int64_t n, const double* coords, int32_t material_id) {
  MPM_GUARD(h)
  if (h->initialised) throw InvalidArg("particles are added before mpm_gpu_initialise");
  auto it = h->mat_index.find(material_id);
  if (it == h->mat_index.end()) throw InvalidArg("unknown material id");
  if (n < 0 || (n > 0 && !coords)) throw InvalidArg("bad particle array");
  if (h->np + n > INT32_MAX) throw InvalidArg("too many particles for 32-bit indices");
  h->p_coords.insert(h->p_coords.end(), coords, coords + n * h->dim);
  h->p_mat.insert(h->p_mat.end(), (size_t)n, (uint16_t)it->second);
  h->set_np(h->np + n);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_assign_particle_materials(mpm_gpu_t h, int64_t n, const int64_t* pids,
                                      int32_t material_id) {
  MPM_GUARD(h)
  if (h->initialised) throw InvalidArg("materials are reassigned before mpm_gpu_initialise");
  auto it = h->mat_index.find(material_id);
  if (it == h->mat_index.end()) throw InvalidArg("unknown material id");
  if (n < 0 || (n > 0 && !pids)) throw InvalidArg("bad particle id array");
  // ids without a particle are skipped (mesh.tcc:1181-1187)
  for (int64_t k = 0; k < n; ++k)
    if (pids[k] >= 0 && pids[k] < h->np) h->p_mat[(size_t)pids[k]] = (uint16_t)it->second;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_initialise(mpm_gpu_t h) {
  MPM_GUARD(h)
  if (!h->mesh_set) throw InvalidArg("set the mesh first");
  if (h->mats.empty()) throw InvalidArg("no material");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int64_t np = h->np;
  std::vector<int32_t> cell(np);
  std::vector<int64_t> count(h->ncells, 0);
  for (int64_t p = 0; p < np; ++p) {
    cell[p] = host_scan(h, &h->p_coords[p * h->dim]);
    if (cell[p] < 0) throw InvalidArg("Particle outside the mesh domain");
    ++count[cell[p]];
  }
  std::vector<double> vol(np), rho(np), mass(np);
  h->p_id.resize(np);
  h->p_nsize.assign((size_t)3 * np, 0.0);
  h->p_acc.assign((size_t)3 * np, 0.0);
  h->aux_dirty = true;
  for (int64_t p = 0; p < np; ++p) {
    const MaterialParams& m = h->mats[h->p_mat[p]];
    h->p_id[p] = (uint64_t)p;
    // Particle::assign_volume (particle.tcc:557-583): unit element length 2
    // over the cell's particle count to the power 1/dim
    const double ns = 2.0 / std::pow((double)count[cell[p]], 1.0 / h->dim);
    for (int d = 0; d < h->dim; ++d) h->p_nsize[(size_t)d * np + p] = ns;
    vol[p] = h->cell_volume[cell[p]] / (double)count[cell[p]];
    rho[p] = m.density;
    mass[p] = vol[p] * rho[p];
  }
  allocate_particles(h);
  upload_pvc(h);
  mpm_gpu_particles in{};
  in.volume = vol.data();
  in.density = rho.data();
  in.mass = mass.data();
  pack_particles(h, &in, &cell);
  refresh_state(h);
  ck(cudaStreamSynchronize(h->stream), "sync");
  h->initialised = true;
  h->step = 0;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_assign_particle_stresses(mpm_gpu_t h, int64_t n, const double* stress) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("No particles have been assigned in mesh, cannot assign stresses");
  if (n != h->np || !stress) throw InvalidArg("Number of particles in mesh and initial stresses don't match");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int dim = h->dim;
  const int S = dim == 2 ? PF<2>::S : PF<3>::S;
  const int ns = dim == 2 ? PF<2>::NS : PF<3>::NS;
  const int64_t npad = h->npad;
  std::vector<double> cols((size_t)ns * npad, 0.0);
  for (int64_t p = 0; p < n; ++p) {
    if (dim == 2 && (stress[p * 6 + 4] != 0. || stress[p * 6 + 5] != 0.))
      throw InvalidArg("2D particle stress must have zero yz and xz components");
    for (int k = 0; k < ns; ++k) cols[(size_t)k * npad + p] = stress[p * 6 + k];
  }
  if (h->mixed) {
    const std::vector<float> colf(cols.begin(), cols.end());
    const int SM = dim == 2 ? PM<2>::S : PM<3>::S;
    ck(cudaMemcpyAsync(h->d_pm.p + (size_t)SM * npad, colf.data(), sizeof(float) * colf.size(),
                       cudaMemcpyHostToDevice, h->stream), "H2D");
    ck(cudaStreamSynchronize(h->stream), "sync");
  } else {
    ck(cudaMemcpyAsync(h->d_pf.p + (size_t)S * npad, cols.data(), sizeof(double) * cols.size(),
                       cudaMemcpyHostToDevice, h->stream), "H2D");
  }
  ck(cudaStreamSynchronize(h->stream), "sync");
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_add_particle_velocity_constraint(mpm_gpu_t h, int64_t n, const int64_t* pids,
                                             int32_t dir, double velocity) {
  MPM_GUARD(h)
  if (dir < 0 || dir >= h->dim) throw InvalidArg("Invalid direction of velocity constraint");
  if (n < 0) {
    for (int64_t p = 0; p < h->np; ++p) h->p_vc[p][(unsigned)dir] = velocity;
  } else {
    for (int64_t i = 0; i < n; ++i) {
      if (pids[i] < 0 || pids[i] >= h->np) throw InvalidArg("particle id out of range");
      h->p_vc[pids[i]][(unsigned)dir] = velocity;
    }
  }
  if (h->initialised) {
    ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
    upload_pvc(h);
    refresh_state(h);
  }
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_load_particles(mpm_gpu_t h, int64_t n, const mpm_gpu_particles* in) {
  MPM_GUARD(h)
  if (!h->mesh_set) throw InvalidArg("set the mesh first");
  if (!in || !in->x || !in->volume || !in->cell || !in->material)
    throw InvalidArg("load_particles needs x, volume, cell and material");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  h->set_np(n);
  h->p_coords.resize(n * h->dim);
  double* pc = h->p_coords.data();
  parallel_for(n * h->dim, [&](int64_t a, int64_t b) { std::fill(pc + a, pc + b, 0.); });
  h->p_mat.resize(n);
  parallel_for(n, [&](int64_t a, int64_t b) {
    int32_t last_id = 0;
    int last_slot = -1;  // runs of one material look the map up once
    for (int64_t p = a; p < b; ++p) {
      const int32_t id = in->material[p];
      if (last_slot < 0 || id != last_id) {
        auto it = h->mat_index.find(id);
        if (it == h->mat_index.end()) throw InvalidArg("unknown material id");
        last_id = id;
        last_slot = it->second;
      }
      h->p_mat[p] = (uint16_t)last_slot;
    }
  });
  h->p_vc.clear();
  h->ntangent = 0;  // a new state has no tangents
  if ((int64_t)h->p_id.size() != n) {
    h->p_id.resize(n);
    for (int64_t p = 0; p < n; ++p) h->p_id[p] = (uint64_t)p;
    h->p_nsize.assign((size_t)3 * n, 0.0);
    h->p_acc.assign((size_t)3 * n, 0.0);
  }
  h->aux_dirty = true;
  allocate_particles(h);
  upload_pvc(h);
  const bool full = in->u && in->v && in->stress && in->strain && in->F && in->mass &&
                    in->density && (!h->any_mc || in->svars);
  if (full)
    load_rows_device(h, in);
  else
    pack_particles(h, in, nullptr);
  refresh_state(h);
  ck(cudaStreamSynchronize(h->stream), "sync");
  h->initialised = true;
  MPM_END(h)
  return MPM_OK;
}

static bool same_step(const DevState& a, const DevState& b, const StepArgs& x, const StepArgs& y) {
  return std::memcmp(&a, &b, sizeof(DevState)) == 0 && x.scheme == y.scheme && x.flip == y.flip && x.vupd == y.vupd &&
         x.remove_lost == y.remove_lost && x.dt == y.dt && x.beta == y.beta &&
         x.damping == y.damping && x.g[0] == y.g[0] && x.g[1] == y.g[1] && x.g[2] == y.g[2] &&
         x.p2g_tile == y.p2g_tile && x.node_threads == y.node_threads &&
         x.return_blocks_per_sm == y.return_blocks_per_sm;
}

// The step arguments of the solver's configuration and launch shape (gravity
// and phase set by the caller).
static StepArgs base_step_args(mpm_gpu_t h) {
  StepArgs a{};
  a.scheme = h->cfg.scheme;
  a.flip = h->cfg.velocity_update == MPM_VELOCITY_FLIP ? 1 : 0;
  a.vupd = h->cfg.velocity_update;
  a.remove_lost = h->cfg.locate_particles ? 0 : 1;
  a.dt = h->cfg.dt;
  a.beta = h->cfg.blending_ratio;
  a.damping = h->cfg.damping_factor;
  a.p2g_tile = h->shape_p2g_tile;
  a.node_threads = h->shape_node_threads;
  a.return_blocks_per_sm = h->shape_return_bps;
  return a;
}

static int run_steps(mpm_gpu_t h, int64_t nsteps, double* elapsed_ms) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("initialise or load particles first");
  if (nsteps < 0) throw InvalidArg("negative step count");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  refresh_state(h);  // constraint or material tables may have been reallocated
  StepArgs a = base_step_args(h);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (elapsed_ms) {
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    ck(cudaEventRecord(e0, h->stream), "cudaEventRecord");
  }
  auto launch = [&]() {
    if (h->ntangent > 0)
      launch_step_tangent(h->dim, h->ds, a, h->stream, h->prof);
    else if (h->mixed)
      launch_step_mixed(h->dim, h->ds, a, h->stream, h->prof);
    else
      launch_step_fp64(h->dim, h->ds, a, h->stream, h->prof);
  };
  if (h->persistent_steps > 0 && !h->prof.enabled) {
    if (!h->structured || h->ntangent > 0)
      return fail(h, MPM_ERR_UNSUPPORTED,
                  "persistent steps need a tensor-product grid and no sensitivities");
    PersistentArgs q{};
    for (int d = 0; d < 3; ++d) q.gravity[d] = d < h->dim ? h->cfg.gravity[d] : 0.;
    q.ramp = h->cfg.gravity_ramping_time;
    q.barrier = h->d_words.p + 4;
    q.step = reinterpret_cast<long long*>(h->d_words.p + 6);
    const long long step_now = h->step;  // each launch advances the device copy
    ck(cudaMemcpyAsync(q.step, &step_now, sizeof(step_now), cudaMemcpyHostToDevice, h->stream), "H2D");
    ck(cudaStreamSynchronize(h->stream), "sync");
    // Launches of persistent_steps steps replay one captured CUDA graph (the
    // barrier reset and the cooperative launch); the first launch of a call
    // and a shorter last one run directly.
    bool eager_done_p = false;
    for (int64_t s = 0; s < nsteps; s += q.nsteps) {
      q.nsteps = std::min<int64_t>(h->persistent_steps, nsteps - s);
      bool launched = false;
      if (q.nsteps == h->persistent_steps && eager_done_p && h->pgraph_ok) {
        if (!(h->pgraph && h->pgraph_steps == q.nsteps && same_step(h->pgraph_state, h->ds, h->pgraph_args, a))) {
          if (h->pgraph) cudaGraphExecDestroy(h->pgraph);
          h->pgraph = nullptr;
          cudaGraph_t g = nullptr;
          bool ok = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
          if (ok) {
            const cudaError_t le = launch_steps_persistent_mixed(h->dim, h->ds, a, q, h->stream);
            ok = cudaStreamEndCapture(h->stream, &g) == cudaSuccess && le == cudaSuccess && g != nullptr;
            ok = ok && cudaGraphInstantiate(&h->pgraph, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
          }
          if (ok) {
            h->pgraph_state = h->ds;
            h->pgraph_args = a;
            h->pgraph_steps = q.nsteps;
          } else {  // no capture of the cooperative launch here: direct launches from now on
            cudaGetLastError();
            if (h->pgraph) cudaGraphExecDestroy(h->pgraph);
            h->pgraph = nullptr;
            h->pgraph_ok = false;
          }
        }
        if (h->pgraph) {
          ck(cudaGraphLaunch(h->pgraph, h->stream), "cudaGraphLaunch");
          launched = true;
        }
      }
      if (!launched) {
        ck(launch_steps_persistent_mixed(h->dim, h->ds, a, q, h->stream), "persistent step launch");
        eager_done_p = true;
      }
      h->prof.launches += 1;
      h->step += q.nsteps;
    }
    nsteps = 0;  // done: the loop below only finishes the call
  }
  // A step whose device state and arguments match the captured one replays the
  // captured CUDA graph (one graph launch instead of the step's kernel
  // launches).  The first step of a call runs eagerly (it sets the kernels'
  // shared-memory attributes outside any capture); profiling runs eagerly.
  bool eager_done = false;
  for (int64_t s = 0; s < nsteps; ++s) {
    double gm = 1.0;  // mpm_explicit.tcc:145-153
    if (h->cfg.gravity_ramping_time > 0.0)
      gm = std::min(1.0, static_cast<double>(h->step) * h->cfg.dt / h->cfg.gravity_ramping_time);
    for (int d = 0; d < 3; ++d) a.g[d] = d < h->dim ? gm * h->cfg.gravity[d] : 0.;
    const bool graphable = h->graph_ok && !h->prof.enabled && eager_done;
    if (graphable && h->graph && same_step(h->graph_state, h->ds, h->graph_args, a)) {
      ck(cudaGraphLaunch(h->graph, h->stream), "cudaGraphLaunch");
      h->prof.launches += h->graph_launches;
    } else if (graphable) {
      if (h->graph) cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
      const int64_t l0 = h->prof.launches;
      cudaGraph_t g = nullptr;
      bool ok = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        launch();
        ok = cudaStreamEndCapture(h->stream, &g) == cudaSuccess && g != nullptr;
        ok = ok && cudaGraphInstantiate(&h->graph, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
      }
      if (ok) {
        h->graph_state = h->ds;
        h->graph_args = a;
        h->graph_launches = h->prof.launches - l0;
        ck(cudaGraphLaunch(h->graph, h->stream), "cudaGraphLaunch");
      } else {  // capture not possible here: launch eagerly from now on
        cudaGetLastError();
        if (h->graph) cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        h->graph_ok = false;
        h->prof.launches = l0;
        launch();
      }
    } else {
      launch();
      eager_done = true;
    }
    ck(cudaGetLastError(), "kernel launch");
    ++h->step;
  }
  if (elapsed_ms) ck(cudaEventRecord(e1, h->stream), "cudaEventRecord");
  unsigned words[2] = {0, 0};
  ck(cudaMemcpyAsync(words, h->d_words.p, sizeof(words), cudaMemcpyDeviceToHost, h->stream), "D2H");
  ck(cudaStreamSynchronize(h->stream), "step");
  h->prof.collect();
  if (elapsed_ms) {
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    *elapsed_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (words[1] & ERR_NONFINITE) return fail(h, MPM_ERR_NONFINITE, "non-finite particle position");
  if (words[1] & ERR_OUTSIDE) return fail(h, MPM_ERR_OUTSIDE, "Particle(s) outside the mesh domain");
  if (words[1] & ERR_BADCELL) return fail(h, MPM_ERR_INVALID, "corrupt particle cell index");
  if (words[1] & ERR_TIMEOUT) return fail(h, MPM_ERR_TIMEOUT, "a bounded device wait (copy, scan or grid barrier) ran out");
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_step(mpm_gpu_t h, int64_t nsteps) { return run_steps(h, nsteps, nullptr); }

int mpm_gpu_step_timed(mpm_gpu_t h, int64_t nsteps, double* elapsed_ms) {
  if (!elapsed_ms) return fail(h, MPM_ERR_INVALID, "null elapsed_ms");
  return run_steps(h, nsteps, elapsed_ms);
}

int mpm_gpu_set_launch_shape(mpm_gpu_t h, int32_t p2g_tile, int32_t node_threads,
                             int32_t return_blocks_per_sm) {
  MPM_GUARD(h)
  if (p2g_tile != 0 && p2g_tile != 128 && p2g_tile != 256)
    throw InvalidArg("p2g_tile must be 0 (default), 128 or 256");
  if (node_threads != 0 && node_threads != 128 && node_threads != 256)
    throw InvalidArg("node_threads must be 0 (default), 128 or 256");
  if (return_blocks_per_sm != 0 && return_blocks_per_sm != 4 && return_blocks_per_sm != 8 &&
      return_blocks_per_sm != 16)
    throw InvalidArg("return_blocks_per_sm must be 0 (default), 4, 8 or 16");
  h->shape_p2g_tile = p2g_tile;
  h->shape_node_threads = node_threads;
  h->shape_return_bps = return_blocks_per_sm;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_set_persistent(mpm_gpu_t h, int32_t steps_per_launch) {
  MPM_GUARD(h)
  if (steps_per_launch < 0) throw InvalidArg("negative steps per launch");
  if (steps_per_launch > 0 &&
      (!h->mixed || h->cfg.scheme != MPM_SCHEME_USL || h->cfg.velocity_update > MPM_VELOCITY_PIC))
    return fail(h, MPM_ERR_UNSUPPORTED, "persistent steps run the mixed USL step with FLIP or PIC");
  h->persistent_steps = steps_per_launch;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_get_persistent(mpm_gpu_t h, int32_t* steps_per_launch, int32_t* graph_replayed) {
  MPM_GUARD(h)
  if (!steps_per_launch || !graph_replayed) throw InvalidArg("null output");
  *steps_per_launch = h->persistent_steps;
  *graph_replayed = h->pgraph != nullptr && h->pgraph_steps == h->persistent_steps ? 1 : 0;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_get_launch_shape(mpm_gpu_t h, int32_t* shape) {
  MPM_GUARD(h)
  if (!shape) throw InvalidArg("null shape");
  const StepArgs a = base_step_args(h);
  shape[0] = tile_threads(a, h->structured);
  shape[1] = node_block(a);
  shape[2] = return_blocks(a);
  MPM_END(h)
  return MPM_OK;
}

// Time each launch-shape candidate on the solver's own state, one field at a
// time (P2G tile, node block, return blocks per SM; each field's best kept
// while the next is tried), restoring the particle state and step counter
// before every trial and at the end.  The launch shape changes no result, so
// the run continues exactly as it would have.
int mpm_gpu_autotune(mpm_gpu_t h, int64_t steps, char* report, size_t report_len) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("initialise or load particles first");
  if (steps < 3) throw InvalidArg("autotune needs at least 3 steps per trial");
  if (h->ntangent > 0) throw InvalidArg("turn sensitivities off first");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  // the state a step changes
  struct Part {
    void* p;
    size_t bytes;
  };
  std::vector<Part> parts = {{h->d_pf.p, h->d_pf.n * sizeof(double)},
                             {h->d_sv.p, h->d_sv.n * sizeof(double)},
                             {h->d_pm.p, h->d_pm.n * sizeof(float)},
                             {h->d_svf.p, h->d_svf.n * sizeof(float)},
                             {h->d_cell.p, h->d_cell.n * sizeof(int32_t)},
                             {h->d_mapb.p, h->d_mapb.n * sizeof(double)},
                             {h->d_rpass.p, h->d_rpass.n * sizeof(uint8_t)}};
  size_t total = 0;
  for (auto& q : parts)
    if (q.p) total += (q.bytes + 255) & ~(size_t)255;
  uint8_t* snap = nullptr;
  if (cudaMalloc(&snap, std::max<size_t>(total, 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(h, MPM_ERR_ALLOC, "autotune needs " + std::to_string(total >> 20) +
                                      " MiB of device memory for a copy of the particle state");
  }
  auto copy = [&](bool save) {
    size_t off = 0;
    for (auto& q : parts) {
      if (!q.p || !q.bytes) continue;
      void* d = save ? (void*)(snap + off) : q.p;
      const void* src = save ? q.p : (const void*)(snap + off);
      ck(cudaMemcpyAsync(d, src, q.bytes, cudaMemcpyDeviceToDevice, h->stream), "D2D");
      off += (q.bytes + 255) & ~(size_t)255;
    }
  };
  const int64_t step0 = h->step;
  const int saved[3] = {h->shape_p2g_tile, h->shape_node_threads, h->shape_return_bps};
  int* field[3] = {&h->shape_p2g_tile, &h->shape_node_threads, &h->shape_return_bps};
  const char* names[3] = {"p2g_tile", "node_threads", "return_blocks_per_sm"};
  const std::vector<int> cand[3] = {
      h->structured ? std::vector<int>{256, 128} : std::vector<int>{128}, {256, 128}, {8, 4, 16}};
  std::string js = "{\"steps_per_trial\": " + std::to_string(steps) + ", \"trials\": {";
  int rc = MPM_OK;
  try {
    copy(true);
    for (int f = 0; f < 3 && rc == MPM_OK; ++f) {
      double best = 1e300;
      int best_v = cand[f][0];
      js += std::string(f ? ", " : "") + "\"" + names[f] + "\": {";
      for (size_t k = 0; k < cand[f].size() && rc == MPM_OK; ++k) {
        *field[f] = cand[f][k];
        copy(false);
        h->step = step0;
        // two untimed steps (an eager one, then the graph capture), then the
        // timed ones (an eager step, then graph replays)
        rc = run_steps(h, 2, nullptr);
        double ms = 0.;
        if (rc == MPM_OK) rc = run_steps(h, steps, &ms);
        js += std::string(k ? ", " : "") + "\"" + std::to_string(cand[f][k]) + "\": " +
              std::to_string(ms / (double)steps);
        if (ms < best) {
          best = ms;
          best_v = cand[f][k];
        }
      }
      js += "}";
      *field[f] = best_v;
    }
    copy(false);
    h->step = step0;
    ck(cudaStreamSynchronize(h->stream), "autotune");
  } catch (...) {
    cudaFree(snap);
    for (int f = 0; f < 3; ++f) *field[f] = saved[f];
    throw;
  }
  cudaFree(snap);
  if (rc != MPM_OK) {  // a trial failed: keep the old shape, report its error
    for (int f = 0; f < 3; ++f) *field[f] = saved[f];
    return rc;
  }
  js += "}, \"chosen\": {\"p2g_tile\": " + std::to_string(h->shape_p2g_tile) +
        ", \"node_threads\": " + std::to_string(h->shape_node_threads) +
        ", \"return_blocks_per_sm\": " + std::to_string(h->shape_return_bps) + "}}";
  if (report && report_len) {
    const size_t n = std::min(js.size(), report_len - 1);
    std::memcpy(report, js.data(), n);
    report[n] = '\0';
  }
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_set_profiling(mpm_gpu_t h, int32_t enable) {
  MPM_GUARD(h)
  h->prof.reset();
  h->prof.enabled = enable != 0;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_kernel_profile(mpm_gpu_t h, int32_t kernel, const char** name, double* total_ms,
                           int64_t* launches) {
  if (!h) return MPM_ERR_INVALID;
  if (kernel < 0 || kernel >= K_NKERNELS) return fail(h, MPM_ERR_INVALID, "kernel index out of range");
  if (name) *name = kernel_name(kernel);
  if (total_ms) *total_ms = h->prof.total_ms[kernel];
  if (launches) *launches = h->prof.count[kernel];
  return MPM_OK;
}

int64_t mpm_gpu_launch_count(mpm_gpu_t h) { return h ? h->prof.launches : -1; }

int64_t mpm_gpu_nparticles(mpm_gpu_t h) { return h ? h->np : -1; }
int64_t mpm_gpu_current_step(mpm_gpu_t h) { return h ? h->step : -1; }

int mpm_gpu_set_isoparametric(mpm_gpu_t h, int32_t isoparametric) {
  MPM_GUARD(h)
  if (h->initialised) throw InvalidArg("set the local-coordinate map before the particles");
  h->isoparametric = isoparametric != 0;
  return MPM_OK;
  MPM_END(h)
}

int mpm_gpu_read_mapping_matrix(mpm_gpu_t h, double* out) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("no particles");
  if (!out) throw InvalidArg("null output");
  if (h->cfg.velocity_update < MPM_VELOCITY_ASFLIP)
    return fail(h, MPM_ERR_UNSUPPORTED, "no mapping matrix: FLIP and PIC carry none");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int dim = h->dim;
  const int64_t np = h->np, ns = h->npad;
  std::vector<double> b((size_t)dim * dim * ns);
  h->d_mapb.download(b.data(), b.size(), h->stream);
  ck(cudaStreamSynchronize(h->stream), "sync");
  for (int64_t p = 0; p < np; ++p)
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c)
        out[p * 9 + a * 3 + c] = (a < dim && c < dim) ? b[(size_t)(a * dim + c) * ns + p] : 0.;
  return MPM_OK;
  MPM_END(h)
}

int mpm_gpu_load_mapping_matrix(mpm_gpu_t h, const double* in) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("no particles");
  if (!in) throw InvalidArg("null input");
  if (h->cfg.velocity_update < MPM_VELOCITY_ASFLIP)
    return fail(h, MPM_ERR_UNSUPPORTED, "no mapping matrix: FLIP and PIC carry none");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int dim = h->dim;
  const int64_t np = h->np, ns = h->npad;
  std::vector<double> b((size_t)dim * dim * ns, 0.0);
  for (int64_t p = 0; p < np; ++p)
    for (int a = 0; a < dim; ++a)
      for (int c = 0; c < dim; ++c) b[(size_t)(a * dim + c) * ns + p] = in[p * 9 + a * 3 + c];
  h->d_mapb.upload(b.data(), b.size(), h->stream);
  ck(cudaStreamSynchronize(h->stream), "sync");
  return MPM_OK;
  MPM_END(h)
}

int mpm_gpu_read_particles(mpm_gpu_t h, mpm_gpu_particles* out) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("no particles");
  if (!out) throw InvalidArg("null output");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int64_t np = h->np;
  std::vector<int32_t> cell(out->cell ? np : 0);
  if (out->cell) h->d_cell.download(cell.data(), np, h->stream);
  // the device writes the requested arrays in the caller's row layout into the
  // staging buffer; one copy each brings them back
  double* const ptr[10] = {out->x, out->u, out->v, out->stress, out->strain, out->F,
                           out->volume, out->mass, out->density, out->svars};
  int64_t total = 0;
  const RowStage r = stage_rows(h, np, ptr, total);
  launch_state_to_rows(h->dim, h->mixed, h->any_mc, h->ds, r, h->stream);
  ck(cudaGetLastError(), "state to rows");
  const int64_t off[10] = {r.x, r.u, r.v, r.stress, r.strain, r.F, r.volume, r.mass, r.density, r.svars};
  const int64_t chunk = std::min(total, ROW_CHUNK);
  if (page_locked(ptr, np)) {
    for (int k = 0; k < 10; ++k)
      if (ptr[k] && np)
        ck(cudaMemcpyAsync(ptr[k], r.base + off[k], sizeof(double) * row_width(k) * np,
                           cudaMemcpyDeviceToHost, h->stream), "D2H");
    ck(cudaStreamSynchronize(h->stream), "sync");
  } else if (double* pin = total ? pinned_rows(h, 2 * chunk) : nullptr) {
    ensure_stage_events(h);
    const int64_t nchunks = (total + chunk - 1) / chunk;
    auto fetch = [&](int64_t c) {  // DMA of chunk c into half c % 2
      const int64_t lo = c * chunk, hi = std::min(total, lo + chunk);
      ck(cudaMemcpyAsync(pin + (c % 2) * chunk, r.base + lo, sizeof(double) * (hi - lo),
                         cudaMemcpyDeviceToHost, h->stream), "D2H");
      ck(cudaEventRecord(h->stage_ev[c % 2], h->stream), "cudaEventRecord");
    };
    for (int64_t c = 0; c < std::min<int64_t>(2, nchunks); ++c) fetch(c);
    for (int64_t c = 0; c < nchunks; ++c) {
      ck(cudaEventSynchronize(h->stage_ev[c % 2]), "row copy");
      const int64_t lo = c * chunk, hi = std::min(total, lo + chunk);
      rows_range(ptr, off, np, lo, hi, pin + (c % 2) * chunk, false);
      if (c + 2 < nchunks) fetch(c + 2);
    }
    ck(cudaStreamSynchronize(h->stream), "sync");
  } else {
    for (int k = 0; k < 10; ++k)
      if (ptr[k] && np)
        ck(cudaMemcpyAsync(ptr[k], r.base + off[k], sizeof(double) * row_width(k) * np,
                           cudaMemcpyDeviceToHost, h->stream), "D2H");
    ck(cudaStreamSynchronize(h->stream), "sync");
  }
  std::vector<int32_t> slot_id(h->mats.size(), -1);  // material slot -> id
  for (auto& kv : h->mat_index) slot_id[kv.second] = kv.first;
  if (out->cell || out->material)
    parallel_for(np, [&](int64_t pa, int64_t pb) {
      for (int64_t p = pa; p < pb; ++p) {
        if (out->cell) out->cell[p] = cell[p];
        if (out->material) out->material[p] = slot_id[h->p_mat[p]];
      }
    });
  MPM_END(h)
  return MPM_OK;
}

}  // extern "C"

namespace {

// PODParticle field sizes (pod_particle.cc dst_sizes): the two bools, the two
// unsigned, everything else 8 bytes
size_t pod_expected_size(int f) {
  if (f == 40 || f == 50) return 1;
  if (f == 52 || f == 53) return 4;
  return 8;
}

void check_pod_layout(size_t record_size, const size_t* offsets, const size_t* sizes,
                      int32_t nfields, PodLayout& L) {
  if (nfields != POD_NFIELDS) throw InvalidArg("a PODParticle record has 74 fields");
  if (!offsets || !sizes) throw InvalidArg("null record layout");
  if (record_size == 0 || record_size % 8 != 0 || record_size > (1u << 16))
    throw InvalidArg("record size must be a positive multiple of 8 bytes");
  for (int f = 0; f < POD_NFIELDS; ++f) {
    if (sizes[f] != pod_expected_size(f))
      throw InvalidArg("PODParticle field " + std::to_string(f) + " has size " +
                       std::to_string(sizes[f]) + ", expected " +
                       std::to_string(pod_expected_size(f)));
    if (offsets[f] % sizes[f] != 0 || offsets[f] + sizes[f] > record_size)
      throw InvalidArg("PODParticle field " + std::to_string(f) +
                       " is misaligned or outside the record");
    L.offset[f] = (int32_t)offsets[f];
  }
  L.record_size = (int64_t)record_size;
}

// Byte runs of a record covered by fields (the rest -- padding, a vtable
// pointer -- is never written into the caller's records).
std::vector<std::pair<size_t, size_t>> pod_runs(const size_t* offsets, const size_t* sizes) {
  std::vector<std::pair<size_t, size_t>> r;
  for (int f = 0; f < POD_NFIELDS; ++f) r.emplace_back(offsets[f], offsets[f] + sizes[f]);
  std::sort(r.begin(), r.end());
  std::vector<std::pair<size_t, size_t>> m;
  for (auto& x : r) {
    if (!m.empty() && x.first <= m.back().second)
      m.back().second = std::max(m.back().second, x.second);
    else
      m.push_back(x);
  }
  return m;
}

void upload_pod_aux(mpm_gpu_t h) {
  if (!h->aux_dirty) return;
  const int64_t np = h->np, ns = h->npad;
  std::vector<uint64_t> id(h->p_id);
  id.resize(ns, 0);
  std::vector<double> nsz((size_t)3 * ns, 0.0), acc((size_t)3 * ns, 0.0);
  for (int d = 0; d < 3; ++d)
    for (int64_t p = 0; p < np; ++p) {
      nsz[(size_t)d * ns + p] = h->p_nsize[(size_t)d * np + p];
      acc[(size_t)d * ns + p] = h->p_acc[(size_t)d * np + p];
    }
  h->d_pid.upload(id.data(), ns, h->stream);
  h->d_nsize.upload(nsz.data(), 3 * ns, h->stream);
  h->d_pacc.upload(acc.data(), 3 * ns, h->stream);
  std::vector<int32_t> ids(h->mats.size(), -1);
  std::vector<uint32_t> nstate(h->mats.size(), 0);
  for (auto& kv : h->mat_index) ids[kv.second] = kv.first;
  for (size_t i = 0; i < h->mats.size(); ++i) nstate[i] = h->mats[i].type == 1 ? SV_N : 0;
  h->d_matid.upload(ids.data(), ids.size(), h->stream);
  h->d_nstate.upload(nstate.data(), nstate.size(), h->stream);
  ck(cudaStreamSynchronize(h->stream), "sync");
  h->aux_dirty = false;
}

// Mesh::locate_particle_cells (mesh.tcc:1116-1151) on the host: the recorded
// cell, its neighbours in ascending id, then every cell in id order.
int32_t host_locate(mpm_gpu_t h, const double* x, int64_t hint) {
  auto inside = [&](int64_t c) {
    double xi[3];
    return host_point_in(h, c, x, xi);
  };
  if (hint >= 0 && hint < h->ncells) {
    if (inside(hint)) return (int32_t)hint;
    if (h->structured) {
      int ijk[3] = {0, 0, 0};
      int64_t c = hint;
      ijk[0] = (int)(c % h->gcells[0]);
      c /= h->gcells[0];
      if (h->dim == 2) {
        ijk[1] = (int)c;
      } else {
        ijk[1] = (int)(c % h->gcells[1]);
        ijk[2] = (int)(c / h->gcells[1]);
      }
      const int kmin = h->dim == 3 ? ijk[2] - 1 : 0, kmax = h->dim == 3 ? ijk[2] + 1 : 0;
      for (int k = kmin; k <= kmax; ++k) {
        if (h->dim == 3 && (k < 0 || k >= h->gcells[2])) continue;
        for (int j = ijk[1] - 1; j <= ijk[1] + 1; ++j) {
          if (j < 0 || j >= h->gcells[1]) continue;
          for (int i = ijk[0] - 1; i <= ijk[0] + 1; ++i) {
            if (i < 0 || i >= h->gcells[0]) continue;
            const int64_t nc = h->dim == 2 ? i + (int64_t)h->gcells[0] * j
                                           : i + (int64_t)h->gcells[0] * (j + (int64_t)h->gcells[1] * k);
            if (nc != hint && inside(nc)) return (int32_t)nc;
          }
        }
      }
    } else {
      for (int32_t k = h->nb_off[hint]; k < h->nb_off[hint + 1]; ++k)
        if (inside(h->nb[k])) return h->nb[k];
    }
  }
  return host_scan(h, x);
}

}  // namespace

extern "C" {

int mpm_gpu_write_pod(mpm_gpu_t h, void* records, int64_t capacity, int64_t* nrecords,
                      size_t record_size, const size_t* offsets, const size_t* sizes,
                      int32_t nfields) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("no particles");
  if (!nrecords) throw InvalidArg("null nrecords");
  PodLayout L{};
  check_pod_layout(record_size, offsets, sizes, nfields, L);
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  refresh_state(h);
  const int64_t np = h->np;
  std::vector<int32_t> cell(np);
  h->d_cell.download(cell.data(), np, h->stream);
  ck(cudaStreamSynchronize(h->stream), "sync");
  std::vector<int32_t> list;
  list.reserve(np);
  for (int64_t p = 0; p < np; ++p)
    if (cell[p] >= 0) list.push_back((int32_t)p);
  const int64_t count = (int64_t)list.size();
  *nrecords = count;
  if (count > capacity) throw InvalidArg("record capacity is below the number of particles in the mesh");
  if (count == 0) return MPM_OK;
  if (!records) throw InvalidArg("null records");
  upload_pod_aux(h);
  h->d_list.upload(list.data(), list.size(), h->stream);
  const auto runs = pod_runs(offsets, sizes);
  // chunks of at most 64 MiB, packed on the device and copied to pinned
  // memory in turn; the host scatters chunk i while the device packs i + 1
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(count, (64 << 20) / (int64_t)record_size));
  const size_t bytes = (size_t)chunk * record_size;
  if (h->d_stage.n < 2 * bytes) h->d_stage.alloc(2 * bytes);
  if (h->h_stage_bytes < 2 * bytes) {
    if (h->h_stage) cudaFreeHost(h->h_stage);
    h->h_stage = nullptr;
    h->h_stage_bytes = 0;
    ck(cudaHostAlloc(reinterpret_cast<void**>(&h->h_stage), 2 * bytes, cudaHostAllocDefault),
       "cudaHostAlloc");
    h->h_stage_bytes = 2 * bytes;
  }
  for (auto& e : h->stage_ev)
    if (!e) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  PodAux a{h->d_pid.p, h->d_nsize.p, h->d_pacc.p, h->d_matid.p, h->d_nstate.p};
  int64_t pend_first[2] = {-1, -1}, pend_n[2] = {0, 0};
  auto drain = [&](int k) {
    if (pend_first[k] < 0) return;
    ck(cudaEventSynchronize(h->stage_ev[k]), "pod copy");
    const uint8_t* src = h->h_stage + (size_t)k * bytes;
    uint8_t* dst = static_cast<uint8_t*>(records) + (size_t)pend_first[k] * record_size;
    for (int64_t i = 0; i < pend_n[k]; ++i)
      for (auto& r : runs)
        std::memcpy(dst + i * record_size + r.first, src + i * record_size + r.first,
                    r.second - r.first);
    pend_first[k] = -1;
  };
  int k = 0;
  for (int64_t first = 0; first < count; first += chunk, k ^= 1) {
    const int64_t n = std::min<int64_t>(chunk, count - first);
    drain(k);
    launch_pod_pack(h->dim, h->mixed, h->ds, a, L, h->d_list.p + first, n,
                    h->d_stage.p + (size_t)k * bytes, h->stream);
    ck(cudaGetLastError(), "pod pack");
    ck(cudaMemcpyAsync(h->h_stage + (size_t)k * bytes, h->d_stage.p + (size_t)k * bytes,
                       (size_t)n * record_size, cudaMemcpyDeviceToHost, h->stream), "D2H");
    ck(cudaEventRecord(h->stage_ev[k], h->stream), "cudaEventRecord");
    pend_first[k] = first;
    pend_n[k] = n;
  }
  drain(k);
  drain(k ^ 1);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_load_pod(mpm_gpu_t h, const void* records, int64_t n, size_t record_size,
                     const size_t* offsets, const size_t* sizes, int32_t nfields) {
  MPM_GUARD(h)
  if (!h->mesh_set) throw InvalidArg("set the mesh first");
  if (h->mats.empty()) throw InvalidArg("no material");
  if (n <= 0 || !records) throw InvalidArg("no records");
  if (n > INT32_MAX) throw InvalidArg("too many particles for 32-bit indices");
  PodLayout L{};
  check_pod_layout(record_size, offsets, sizes, nfields, L);
  const int dim = h->dim;
  const uint8_t* base = static_cast<const uint8_t*>(records);
  auto dbl = [&](int64_t i, int f) {
    double v;
    std::memcpy(&v, base + i * record_size + offsets[f], 8);
    return v;
  };
  auto u64 = [&](int64_t i, int f) {
    uint64_t v;
    std::memcpy(&v, base + i * record_size + offsets[f], 8);
    return v;
  };
  auto u32 = [&](int64_t i, int f) {
    uint32_t v;
    std::memcpy(&v, base + i * record_size + offsets[f], 4);
    return v;
  };
  std::vector<double> x(3 * n), u(3 * n), v(3 * n), st(6 * n), sn(6 * n), F(9 * n), vol(n),
      mass(n), rho(n), sv((size_t)SV_N * n, 0.0);
  std::vector<int64_t> cell(n);
  std::vector<int32_t> mat(n);
  std::vector<uint64_t> ids(n);
  std::vector<double> nsize((size_t)3 * n, 0.0), acc((size_t)3 * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    ids[i] = u64(i, 0);
    mass[i] = dbl(i, 1);
    vol[i] = dbl(i, 2);
    if (!(vol[i] > 0.)) throw InvalidArg("Particle volume cannot be negative");
    rho[i] = mass[i] / vol[i];  // particle.tcc:46-47
    for (int d = 0; d < 3; ++d) {
      const bool in = d < dim;
      x[i * 3 + d] = in ? dbl(i, 4 + d) : 0.;
      u[i * 3 + d] = in ? dbl(i, 7 + d) : 0.;
      v[i * 3 + d] = in ? dbl(i, 13 + d) : 0.;
      if (in) {
        nsize[(size_t)d * n + i] = dbl(i, 10 + d);
        acc[(size_t)d * n + i] = dbl(i, 16 + d);
      }
    }
    for (int k = 0; k < 6; ++k) {
      st[i * 6 + k] = dbl(i, 19 + k);
      sn[i * 6 + k] = dbl(i, 25 + k);
    }
    for (int k = 0; k < 9; ++k) F[i * 9 + k] = dbl(i, 31 + k);
    if (dim == 2) {  // the 2D state has no out-of-plane components
      st[i * 6 + 4] = st[i * 6 + 5] = 0.;
      sn[i * 6 + 2] = sn[i * 6 + 4] = sn[i * 6 + 5] = 0.;
    }
    const uint32_t mid = u32(i, 52);
    auto it = h->mat_index.find((int32_t)mid);
    if (it == h->mat_index.end()) throw InvalidArg("Material is invalid to assign to particle!");
    mat[i] = (int32_t)mid;
    const MaterialParams& m = h->mats[it->second];
    double s9[SV_N] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (m.type == 1) {
      mc_init_state(m, s9);
      if (u32(i, 53) == (uint32_t)SV_N)  // particle.tcc:160-168
        for (int k = 0; k < SV_N; ++k) s9[k] = dbl(i, 54 + k);
    }
    for (int k = 0; k < SV_N; ++k) sv[i * SV_N + k] = s9[k];
    const uint64_t c = u64(i, 51);
    cell[i] = host_locate(h, &x[i * 3], c < (uint64_t)h->ncells ? (int64_t)c : -1);
    if (cell[i] < 0) throw InvalidArg("Particle outside the mesh domain");
  }
  mpm_gpu_particles in{};
  in.x = x.data();
  in.u = u.data();
  in.v = v.data();
  in.stress = st.data();
  in.strain = sn.data();
  in.F = F.data();
  in.volume = vol.data();
  in.mass = mass.data();
  in.density = rho.data();
  in.cell = cell.data();
  in.material = mat.data();
  in.svars = sv.data();
  const int rc = mpm_gpu_load_particles(h, n, &in);
  if (rc != MPM_OK) return rc;
  h->p_id = std::move(ids);
  h->p_nsize = std::move(nsize);
  h->p_acc = std::move(acc);
  h->aux_dirty = true;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_set_sensitivities(mpm_gpu_t h, int32_t n, const int32_t* material_ids,
                              const int32_t* kinds) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("initialise or load particles first");
  if (n < 0 || n > MAX_TANGENTS) throw InvalidArg("at most 2 parameters are differentiated");
  if (n > 0 && (!material_ids || !kinds)) throw InvalidArg("null parameter list");
  if (n > 0 && h->mixed) return fail(h, MPM_ERR_UNSUPPORTED, "sensitivities run in FP64 only");
  if (n > 0 && h->cfg.scheme != MPM_SCHEME_USL)
    return fail(h, MPM_ERR_UNSUPPORTED, "sensitivities follow the USL scheme only");
  if (n > 0 && h->cfg.velocity_update >= MPM_VELOCITY_ASFLIP)
    return fail(h, MPM_ERR_UNSUPPORTED, "sensitivities follow the FLIP and PIC updates only");
  if (n > 0 && h->isoparametric && !h->structured)
    return fail(h, MPM_ERR_UNSUPPORTED, "sensitivities take Cartesian local coordinates only");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  std::vector<TangentParam> params(n);
  for (int k = 0; k < n; ++k) {
    auto it = h->mat_index.find(material_ids[k]);
    if (it == h->mat_index.end()) throw InvalidArg("unknown material id");
    if (kinds[k] < TP_YOUNGS_MODULUS || kinds[k] > TP_DILATION) throw InvalidArg("unknown parameter kind");
    if (kinds[k] != TP_YOUNGS_MODULUS && h->mats[it->second].type != 1)
      throw InvalidArg("friction, cohesion and dilation are MohrCoulomb parameters");
    params[k] = TangentParam{it->second, kinds[k]};
  }
  h->ntangent = 0;
  if (n == 0) {
    refresh_state(h);
    return MPM_OK;
  }
  const int64_t np = h->npad;
  const int nval = 1 + 3 * h->dim;
  if (h->any_mc) h->d_tpbuf.alloc((size_t)7 * (1 + MAX_TANGENTS) * np);
  for (int k = 0; k < MAX_TANGENTS; ++k) {
    h->d_pft[k].alloc((size_t)h->nfields() * np);
    h->d_nft[k].alloc((size_t)h->nnf() * h->nnodes);
    h->d_partt[k].alloc((size_t)h->ncells * h->nv * nval);
    ck(cudaMemsetAsync(h->d_pft[k].p, 0, sizeof(double) * h->nfields() * np, h->stream), "memset");
    ck(cudaMemsetAsync(h->d_nft[k].p, 0, sizeof(double) * h->nnf() * h->nnodes, h->stream), "memset");
    h->d_svt[k].free();
  }
  // material tables and the initial state-variable derivatives
  std::vector<unsigned char> mt(tangent_material_bytes() * h->mats.size());
  std::vector<double> seed((size_t)h->mats.size() * SV_N * MAX_TANGENTS);
  make_tangent_materials(h->mats.data(), (int)h->mats.size(), params.data(), n, mt.data(),
                         seed.data());
  h->d_mats_t.upload(mt.data(), mt.size(), h->stream);
  if (h->any_mc) {
    for (int k = 0; k < MAX_TANGENTS; ++k) {
      std::vector<double> svt((size_t)SV_N * np, 0.0);
      for (int64_t p = 0; p < h->np; ++p)
        for (int v = 0; v < SV_N; ++v)
          svt[(size_t)v * np + p] = seed[((size_t)h->p_mat[p] * SV_N + v) * MAX_TANGENTS + k];
      h->d_svt[k].upload(svt.data(), svt.size(), h->stream);
    }
  }
  ck(cudaStreamSynchronize(h->stream), "sync");
  // nodes below 1e-3 of the mean particle mass pass no derivatives
  {
    std::vector<double> mass(h->np);
    const int MASSF = h->dim == 2 ? PF<2>::MASS : PF<3>::MASS;
    ck(cudaMemcpy(mass.data(), h->d_pf.p + (size_t)MASSF * h->npad, sizeof(double) * h->np,
                  cudaMemcpyDeviceToHost), "D2H");
    double sum = 0.0;
    for (double v : mass) sum += v;
    h->tangent_mass_floor = h->np > 0 ? 1e-3 * sum / (double)h->np : 0.0;
  }
  h->ntangent = n;
  refresh_state(h);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_read_sensitivities(mpm_gpu_t h, int32_t field, double* out) {
  MPM_GUARD(h)
  if (h->ntangent == 0) throw InvalidArg("no sensitivities enabled");
  if (!out) throw InvalidArg("null output");
  const int dim = h->dim;
  int off = 0, nc = 0;
  switch (field) {
    case 0: off = dim == 2 ? PF<2>::X : PF<3>::X; nc = dim; break;
    case 1: off = dim == 2 ? PF<2>::U : PF<3>::U; nc = dim; break;
    case 2: off = dim == 2 ? PF<2>::V : PF<3>::V; nc = dim; break;
    case 3: off = dim == 2 ? PF<2>::S : PF<3>::S; nc = dim == 2 ? 4 : 6; break;
    default: throw InvalidArg("field: 0 x, 1 u, 2 v, 3 stress");
  }
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int64_t np = h->np, ns = h->npad;
  const int width = field == 3 ? 6 : 3;
  std::vector<double> col((size_t)nc * ns);
  for (int k = 0; k < h->ntangent; ++k) {
    ck(cudaMemcpyAsync(col.data(), h->d_pft[k].p + (size_t)off * ns, sizeof(double) * nc * ns,
                       cudaMemcpyDeviceToHost, h->stream), "D2H");
    ck(cudaStreamSynchronize(h->stream), "sync");
    double* o = out + (size_t)k * np * width;
    for (int64_t p = 0; p < np; ++p)
      for (int c = 0; c < width; ++c) o[p * width + c] = c < nc ? col[(size_t)c * ns + p] : 0.0;
  }
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_set_current_step(mpm_gpu_t h, int64_t step) {
  MPM_GUARD(h)
  if (step < 0) throw InvalidArg("negative step");
  h->step = step;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_device_field(mpm_gpu_t h, int32_t field, void** base, int64_t* stride, int32_t* ncomp) {
  MPM_GUARD(h)
  if (!h->initialised || !base || !stride || !ncomp) throw InvalidArg("bad call");
  const int dim = h->dim;
  if (h->mixed && field != 0 && field != 1)
    return fail(h, MPM_ERR_UNSUPPORTED, "mixed precision: only x and u are FP64 device fields");
  int off = 0, nc = 0;
  switch (field) {
    case 0: off = dim == 2 ? PF<2>::X : PF<3>::X; nc = dim; break;
    case 1: off = dim == 2 ? PF<2>::U : PF<3>::U; nc = dim; break;
    case 2: off = dim == 2 ? PF<2>::V : PF<3>::V; nc = dim; break;
    case 3: off = dim == 2 ? PF<2>::S : PF<3>::S; nc = dim == 2 ? 4 : 6; break;
    case 4: off = dim == 2 ? PF<2>::E : PF<3>::E; nc = dim == 2 ? 3 : 6; break;
    case 5: off = dim == 2 ? PF<2>::F : PF<3>::F; nc = dim == 2 ? 4 : 9; break;
    case 6: off = dim == 2 ? PF<2>::VOL : PF<3>::VOL; nc = 1; break;
    case 7: off = dim == 2 ? PF<2>::RHO : PF<3>::RHO; nc = 1; break;
    case 8: off = dim == 2 ? PF<2>::MASS : PF<3>::MASS; nc = 1; break;
    default: throw InvalidArg("unknown field");
  }
  *base = h->d_pf.p + (size_t)off * h->npad;
  *stride = h->npad;
  *ncomp = nc;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_material_stress_batch(int32_t device, int32_t dim, const char* type,
                                  const char* json_props, int64_t n, const double* stress,
                                  const double* dstrain, const double* density, double* state,
                                  double* out) {
  if (dim != 2 && dim != 3) return MPM_ERR_INVALID;
  if (n < 0 || !type || !json_props || (n > 0 && (!stress || !dstrain || !density || !state || !out)))
    return MPM_ERR_INVALID;
  try {
    const MaterialParams m = make_material(dim, type, parse_json(json_props));
    ck(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t st;
    ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    DevBuf<double> ds, dd, dr, dv, dout;
    ds.upload(stress, n * 6, st);
    dd.upload(dstrain, n * 6, st);
    dr.upload(density, n, st);
    dv.upload(state, n * SV_N, st);
    dout.alloc(std::max<int64_t>(1, n * 6));
    launch_material_batch_fp64(dim, n, m, ds.p, dd.p, dr.p, dv.p, dout.p, st);
    ck(cudaGetLastError(), "launch");
    dout.download(out, n * 6, st);
    dv.download(state, n * SV_N, st);
    ck(cudaStreamSynchronize(st), "sync");
    cudaStreamDestroy(st);
  } catch (const InvalidArg&) {
    return MPM_ERR_INVALID;
  } catch (const CudaError&) {
    return MPM_ERR_CUDA;
  } catch (const std::exception&) {
    return MPM_ERR_INVALID;
  }
  return MPM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ adjoint
namespace {


// gravity of solver step `step` (the ramp of mpm_explicit.tcc:145-153, as run_steps)
void set_gravity(mpm_gpu_t h, StepArgs& a, int64_t step) {
  double gm = 1.0;
  if (h->cfg.gravity_ramping_time > 0.0)
    gm = std::min(1.0, static_cast<double>(step) * h->cfg.dt / h->cfg.gravity_ramping_time);
  for (int d = 0; d < 3; ++d) a.g[d] = d < h->dim ? gm * h->cfg.gravity[d] : 0.;
}

// Save the solver's particle state to (pf, sv, cell) or restore it from there:
// the whole FP64 particle buffer (full), or the compact rows of t.range one
// after another.
void copy_state(mpm_gpu_t h, const AdjointTape& t, double* pf, double* sv, int32_t* cell, bool save,
                bool full = false) {
  auto cp = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream), "D2D");
  };
  if (full) {
    if (save)
      cp(pf, h->d_pf.p, t.pf_n * sizeof(double));
    else
      cp(h->d_pf.p, pf, t.pf_n * sizeof(double));
  } else {
    const size_t np = (size_t)h->npad;
    size_t at = 0;
    for (int r = 0; r < t.nranges; ++r) {
      const size_t n = (size_t)(t.range[r][1] - t.range[r][0]) * np;
      double* dev = h->d_pf.p + (size_t)t.range[r][0] * np;
      if (save)
        cp(pf + at, dev, n * sizeof(double));
      else
        cp(dev, pf + at, n * sizeof(double));
      at += n;
    }
  }
  if (save) {
    cp(sv, h->d_sv.p, t.sv_n * sizeof(double));
    cp(cell, h->d_cell.p, t.cell_n * sizeof(int32_t));
  } else {
    cp(h->d_sv.p, sv, t.sv_n * sizeof(double));
    cp(h->d_cell.p, cell, t.cell_n * sizeof(int32_t));
  }
}

}  // namespace

extern "C" {

int mpm_gpu_adjoint_record(mpm_gpu_t h, int64_t nsteps, int64_t checkpoint_every, int32_t nparams,
                           const int32_t* material_ids, const int32_t* kinds) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("initialise or load particles first");
  if (nsteps < 1 || checkpoint_every < 0)
    throw InvalidArg("nsteps must be >= 1 and checkpoint_every >= 0 (0: chosen by the library)");
  if (nparams < 0 || nparams > MAX_TANGENTS) throw InvalidArg("at most 2 parameters");
  if (nparams > 0 && (!material_ids || !kinds)) throw InvalidArg("null parameter list");
  if (h->mixed) return fail(h, MPM_ERR_UNSUPPORTED, "the adjoint runs in FP64 only");
  if (h->cfg.scheme != MPM_SCHEME_USL)
    return fail(h, MPM_ERR_UNSUPPORTED, "the adjoint follows the USL scheme only");
  if (h->cfg.velocity_update >= MPM_VELOCITY_ASFLIP)
    return fail(h, MPM_ERR_UNSUPPORTED, "the adjoint follows the FLIP and PIC updates only");
  if (!h->structured)
    return fail(h, MPM_ERR_UNSUPPORTED, "the adjoint runs on tensor-product grids (box cells) only");
  if (h->ds.any_softening)
    return fail(h, MPM_ERR_UNSUPPORTED, "the adjoint does not differentiate softening materials");
  if (h->ntangent > 0) return fail(h, MPM_ERR_UNSUPPORTED, "turn sensitivities off first");
  std::vector<TangentParam> params(nparams);
  for (int k = 0; k < nparams; ++k) {
    auto it = h->mat_index.find(material_ids[k]);
    if (it == h->mat_index.end()) throw InvalidArg("unknown material id");
    if (kinds[k] < TP_YOUNGS_MODULUS || kinds[k] > TP_DILATION) throw InvalidArg("unknown parameter kind");
    if (kinds[k] != TP_YOUNGS_MODULUS && h->mats[it->second].type != 1)
      throw InvalidArg("friction, cohesion and dilation are MohrCoulomb parameters");
    params[k] = TangentParam{it->second, kinds[k]};
  }
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  // a tape of an earlier record keeps its buffers: a calibration loop records
  // and reverses the same run shape again and again
  if (!h->tape) h->tape.reset(new AdjointTape());
  AdjointTape& t = *h->tape;
  t.recorded = false;
  const size_t held = t.ck_pf.n * 8 + t.ck_sv.n * 8 + t.ck_cell.n * 4 + t.seg_pf.n * 8 +
                      t.seg_sv.n * 8 + t.seg_cell.n * 4 + t.fin_pf.n * 8 + t.fin_sv.n * 8 +
                      t.fin_cell.n * 4 + (t.adj.n + t.deps.n + t.dsbar.n + t.coef.n + t.theta.n +
                                          t.apart.n + t.nbar.n) * 8;
  t.nsteps = nsteps;
  t.nparams = nparams;
  t.np = h->np;
  t.pf_n = h->d_pf.n;
  {
    const bool d3 = h->dim == 3;
    const int X = d3 ? PF<3>::X : PF<2>::X, V = d3 ? PF<3>::V : PF<2>::V,
              S = d3 ? PF<3>::S : PF<2>::S, NS = d3 ? PF<3>::NS : PF<2>::NS,
              VOL = d3 ? PF<3>::VOL : PF<2>::VOL, MASS = d3 ? PF<3>::MASS : PF<2>::MASS;
    static_assert(PF<3>::V + 3 == PF<3>::S && PF<2>::V + 2 == PF<2>::S, "v then stress");
    static_assert(PF<3>::VOL + 1 == PF<3>::RHO && PF<3>::RHO + 1 == PF<3>::MASS, "V, rho, m");
    static_assert(PF<2>::VOL + 1 == PF<2>::RHO && PF<2>::RHO + 1 == PF<2>::MASS, "V, rho, m");
    const int rg[3][2] = {{X, X + h->dim}, {V, S + NS}, {VOL, MASS + 1}};
    t.nranges = 3;
    t.pfc_n = 0;
    for (int r = 0; r < 3; ++r) {
      t.range[r][0] = rg[r][0];
      t.range[r][1] = rg[r][1];
      t.pfc_n += (size_t)(rg[r][1] - rg[r][0]) * (size_t)h->npad;
    }
  }
  t.sv_n = h->d_sv.n;
  t.cell_n = h->d_cell.n;
  const int dim = h->dim;
  const int64_t np = h->npad;
  const int ns = dim == 2 ? PF<2>::NS : PF<3>::NS;
  const size_t state_bytes = t.pfc_n * 8 + t.sv_n * 8 + t.cell_n * 4;  // a compact state
  const size_t work_bytes = (size_t)np * 8 * ((2 * dim + ns + 1) + 6 + ns + (3 * dim + 6) + MAX_TANGENTS) +
                            (size_t)h->ncells * h->nv * 2 * dim * 8 + (size_t)h->nnodes * (1 + 3 * dim) * 8;
  const size_t end_bytes = t.pf_n * 8 + t.sv_n * 8 + t.cell_n * 4;  // the whole end state
  auto need_for = [&](int64_t every) {
    const int64_t nck = (nsteps + every - 1) / every;
    return state_bytes * (size_t)(nck + std::min(every, nsteps)) + end_bytes + work_bytes;
  };
  size_t free_b = 0, total_b = 0;
  ck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  free_b += held;  // the tape's own buffers count as available
  if (checkpoint_every == 0) {
    // every step's start state kept when half the free memory holds them (the
    // reverse sweep then recomputes nothing), else checkpoints sqrt(nsteps)
    // apart, the least memory
    checkpoint_every = 1;
    if (need_for(1) > free_b / 2)
      checkpoint_every = std::max<int64_t>(1, (int64_t)std::ceil(std::sqrt((double)nsteps)));
  }
  t.every = checkpoint_every;
  const int64_t nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  const int64_t nseg = std::min(checkpoint_every, nsteps);
  const size_t need = need_for(checkpoint_every);
  if (need > free_b) {
    h->tape.reset();
    return fail(h, MPM_ERR_ALLOC, "the adjoint needs " + std::to_string(need >> 20) + " MiB (" +
                                      std::to_string(nck) + " checkpoints and " + std::to_string(nseg) +
                                      " segment states); " + std::to_string(free_b >> 20) +
                                      " MiB are free: raise checkpoint_every towards sqrt(nsteps)");
  }
  t.ck_pf.resize(t.pfc_n * nck);
  t.ck_sv.resize(t.sv_n * nck);
  t.ck_cell.resize(t.cell_n * nck);
  t.seg_pf.resize(t.pfc_n * nseg);
  t.seg_sv.resize(t.sv_n * nseg);
  t.seg_cell.resize(t.cell_n * nseg);
  t.fin_pf.resize(t.pf_n);
  t.fin_sv.resize(t.sv_n);
  t.fin_cell.resize(t.cell_n);
  t.adj.resize((size_t)(2 * dim + ns + 1) * np);
  t.deps.resize((size_t)6 * np);
  t.dsbar.resize((size_t)ns * np);
  t.coef.resize((size_t)(3 * dim + 6) * np);
  t.theta.resize((size_t)MAX_TANGENTS * np);
  t.apart.resize((size_t)h->ncells * h->nv * 2 * dim);
  t.nbar.resize((size_t)(1 + 3 * dim) * h->nnodes);
  // Dual materials: zero derivatives (the return map's Jacobian) and the
  // parameters' derivatives, with the initial state's parameter derivatives
  {
    std::vector<unsigned char> mz(tangent_material_bytes() * h->mats.size()),
        mp(tangent_material_bytes() * h->mats.size());
    std::vector<double> seed0((size_t)h->mats.size() * SV_N * MAX_TANGENTS),
        seed((size_t)h->mats.size() * SV_N * MAX_TANGENTS);
    make_tangent_materials(h->mats.data(), (int)h->mats.size(), nullptr, 0, mz.data(), seed0.data());
    make_tangent_materials(h->mats.data(), (int)h->mats.size(), params.data(), nparams, mp.data(),
                           seed.data());
    t.mats_zero.upload(mz.data(), mz.size(), h->stream);
    t.mats_param.upload(mp.data(), mp.size(), h->stream);
    t.sv_seed.upload(seed.data(), seed.size(), h->stream);
  }
  // nodes below 1e-3 of the mean particle mass pass no cotangents (the
  // tangent step's rule, so the two gradients are the same derivative)
  {
    std::vector<double> mass(h->np);
    const int MASSF = dim == 2 ? PF<2>::MASS : PF<3>::MASS;
    ck(cudaMemcpyAsync(mass.data(), h->d_pf.p + (size_t)MASSF * np, sizeof(double) * h->np,
                       cudaMemcpyDeviceToHost, h->stream), "D2H");
    ck(cudaStreamSynchronize(h->stream), "sync");
    double sum = 0.0;
    for (double v : mass) sum += v;
    t.mass_floor = h->np > 0 ? 1e-3 * sum / (double)h->np : 0.0;
  }
  t.step0 = h->step;
  for (int64_t s0 = 0; s0 < nsteps; s0 += checkpoint_every) {
    const int64_t k = s0 / checkpoint_every;
    copy_state(h, t, t.ck_pf.p + t.pfc_n * k, t.ck_sv.p + t.sv_n * k, t.ck_cell.p + t.cell_n * k, true);
    const int rc = run_steps(h, std::min(checkpoint_every, nsteps - s0), nullptr);
    if (rc != MPM_OK) {
      h->tape.reset();
      return rc;
    }
  }
  t.recorded = true;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_adjoint_reverse(mpm_gpu_t h, const double* dL_dx, const double* dL_dv,
                            double* dL_dparams, double* dL_dx0, double* dL_dv0,
                            double* dL_dstress0) {
  MPM_GUARD(h)
  if (!h->tape || !h->tape->recorded) throw InvalidArg("record a forward run first (mpm_gpu_adjoint_record)");
  AdjointTape& t = *h->tape;
  if (h->step != t.step0 + t.nsteps || h->np != t.np || h->d_pf.n != t.pf_n)
    throw InvalidArg("the state changed since the recorded run");
  if (!dL_dx && !dL_dv) throw InvalidArg("no terminal cotangent (dL_dx and dL_dv are both null)");
  if (t.nparams > 0 && !dL_dparams) throw InvalidArg("null dL_dparams");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int dim = h->dim;
  const int64_t np = h->npad, n = h->np;
  const int ns = dim == 2 ? PF<2>::NS : PF<3>::NS;
  const int AX = 0, AV = dim, AS = 2 * dim, AVOL = 2 * dim + ns, AN = 2 * dim + ns + 1;
  copy_state(h, t, t.fin_pf.p, t.fin_sv.p, t.fin_cell.p, true, true);
  {  // terminal cotangents, rows -> the device layout
    std::vector<double> a((size_t)AN * np, 0.0);
    for (int64_t p = 0; p < n; ++p)
      for (int d = 0; d < dim; ++d) {
        if (dL_dx) a[(size_t)(AX + d) * np + p] = dL_dx[p * 3 + d];
        if (dL_dv) a[(size_t)(AV + d) * np + p] = dL_dv[p * 3 + d];
      }
    t.adj.upload(a.data(), a.size(), h->stream);
    ck(cudaMemsetAsync(t.theta.p, 0, sizeof(double) * t.theta.n, h->stream), "memset");
    ck(cudaStreamSynchronize(h->stream), "sync");
  }
  AdjointArgs A;
  A.adj = t.adj.p;
  A.deps = t.deps.p;
  A.dsbar = t.dsbar.p;
  A.coef = t.coef.p;
  A.theta = t.theta.p;
  A.apart = t.apart.p;
  A.nbar = t.nbar.p;
  A.mats_zero = t.mats_zero.p;
  A.mats_param = t.mats_param.p;
  A.sv_seed = t.sv_seed.p;
  A.nparams = t.nparams;
  A.mass_floor = t.mass_floor;
  StepArgs a = base_step_args(h);
  refresh_state(h);
  const int64_t nck = (t.nsteps + t.every - 1) / t.every;
  for (int64_t seg = nck - 1; seg >= 0; --seg) {
    const int64_t s0 = seg * t.every, s1 = std::min(s0 + t.every, t.nsteps);
    copy_state(h, t, t.ck_pf.p + t.pfc_n * seg, t.ck_sv.p + t.sv_n * seg, t.ck_cell.p + t.cell_n * seg,
               false);
    for (int64_t k = s0; k < s1 - 1; ++k) {  // the segment's step-start states
      const int64_t j = k - s0;
      copy_state(h, t, t.seg_pf.p + t.pfc_n * j, t.seg_sv.p + t.sv_n * j, t.seg_cell.p + t.cell_n * j, true);
      set_gravity(h, a, t.step0 + k);
      launch_step_fp64(dim, h->ds, a, h->stream, h->prof);
    }
    // the device state is now the last step's start: reversed first, with no copy
    for (int64_t k = s1 - 1; k >= s0; --k) {
      const int64_t j = k - s0;
      if (k < s1 - 1)
        copy_state(h, t, t.seg_pf.p + t.pfc_n * j, t.seg_sv.p + t.sv_n * j, t.seg_cell.p + t.cell_n * j,
                   false);
      set_gravity(h, a, t.step0 + k);
      h->prof.begin(K_ADJ_RECOMPUTE, h->stream, SORT_KERNELS + 2);
      launch_p2g_nodes_fp64(dim, h->ds, a, h->stream);
      h->prof.end(K_ADJ_RECOMPUTE, h->stream);
      launch_adjoint_step(dim, h->ds, A, a, h->stream, h->prof);
    }
    ck(cudaGetLastError(), "adjoint launch");
  }
  std::vector<double> adj((size_t)AN * np), theta((size_t)MAX_TANGENTS * np);
  t.adj.download(adj.data(), adj.size(), h->stream);
  t.theta.download(theta.data(), theta.size(), h->stream);
  unsigned words[2] = {0, 0};
  ck(cudaMemcpyAsync(words, h->d_words.p, sizeof(words), cudaMemcpyDeviceToHost, h->stream), "D2H");
  // back to the recorded run's end state
  copy_state(h, t, t.fin_pf.p, t.fin_sv.p, t.fin_cell.p, false, true);
  ck(cudaStreamSynchronize(h->stream), "adjoint");
  h->prof.collect();
  if (words[1] & ERR_NONFINITE) return fail(h, MPM_ERR_NONFINITE, "non-finite state in the recomputed run");
  if (words[1] & ERR_TIMEOUT) return fail(h, MPM_ERR_TIMEOUT, "a bounded device wait (copy, scan or grid barrier) ran out");
  for (int q = 0; q < t.nparams; ++q) {  // particle order: a fixed summation order
    double sum = 0.0;
    for (int64_t p = 0; p < n; ++p) sum += theta[(size_t)q * np + p];
    dL_dparams[q] = sum;
  }
  for (int64_t p = 0; p < n; ++p) {
    for (int d = 0; d < 3; ++d) {
      if (dL_dx0) dL_dx0[p * 3 + d] = d < dim ? adj[(size_t)(AX + d) * np + p] : 0.0;
      if (dL_dv0) dL_dv0[p * 3 + d] = d < dim ? adj[(size_t)(AV + d) * np + p] : 0.0;
    }
    if (dL_dstress0)
      for (int k = 0; k < 6; ++k) dL_dstress0[p * 6 + k] = k < ns ? adj[(size_t)(AS + k) * np + p] : 0.0;
  }
  (void)AVOL;
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_adjoint_run(mpm_gpu_t h, int64_t nsteps, int64_t checkpoint_every, int32_t nparams,
                        const int32_t* material_ids, const int32_t* kinds, const double* x_target,
                        double* loss, double* dL_dparams) {
  if (!h) return MPM_ERR_INVALID;
  if (!x_target || !loss) return fail(h, MPM_ERR_INVALID, "null x_target or loss");
  int rc = mpm_gpu_adjoint_record(h, nsteps, checkpoint_every, nparams, material_ids, kinds);
  if (rc != MPM_OK) return rc;
  std::vector<double> g;  // dL/dx at the end of the run
  MPM_GUARD(h)
  const int dim = h->dim;
  const int64_t np = h->npad, n = h->np;
  std::vector<double> x((size_t)dim * np);
  const int XF = 0;  // PF<DIM>::X
  ck(cudaMemcpyAsync(x.data(), h->d_pf.p + (size_t)XF * np, sizeof(double) * dim * np,
                     cudaMemcpyDeviceToHost, h->stream), "D2H");
  std::vector<int32_t> cell(np);
  ck(cudaMemcpyAsync(cell.data(), h->d_cell.p, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, h->stream), "D2H");
  ck(cudaStreamSynchronize(h->stream), "sync");
  g.assign((size_t)n * 3, 0.0);
  double L = 0.0;
  for (int64_t p = 0; p < n; ++p) {
    if (cell[p] < 0) continue;  // removed particles are not in the loss
    for (int d = 0; d < dim; ++d) {
      const double r = x[(size_t)d * np + p] - x_target[p * 3 + d];
      L += r * r;
      g[p * 3 + d] = 2.0 * r;
    }
  }
  *loss = L;
  MPM_END(h)
  return mpm_gpu_adjoint_reverse(h, g.data(), nullptr, dL_dparams, nullptr, nullptr, nullptr);
}

}  // extern "C"

// ------------------------------------------------------------ HDF5 particle table
namespace {

// The reference's PODParticle (pod_particle.h:12-62) as its compiler lays it
// out: a vtable pointer first (the struct has a virtual destructor), then the
// data members at natural alignment; 592 bytes.  Field names and HDF5 types of
// pod_particle.cc (id and cell_id H5T_NATIVE_LLONG, the two flags
// H5T_NATIVE_HBOOL, material_id and nstate_vars H5T_NATIVE_UINT).
struct RefPod {
  size_t size = 592;
  std::vector<std::string> names;
  std::vector<const char*> cnames;
  size_t off[POD_NFIELDS], sz[POD_NFIELDS];
  int32_t type[POD_NFIELDS];
  RefPod() {
    size_t o = 8;  // vtable pointer
    int f = 0;
    auto add = [&](const std::string& n, size_t s, int t) {
      o = (o + s - 1) / s * s;
      names.push_back(n);
      off[f] = o;
      sz[f] = s;
      type[f] = t;
      o += s;
      ++f;
    };
    add("id", 8, MPM_H5_I64);
    for (const char* n : {"mass", "volume", "pressure"}) add(n, 8, MPM_H5_F64);
    for (const char* v : {"coord", "displacement", "nsize", "velocity", "acceleration"})
      for (const char* c : {"_x", "_y", "_z"}) add(std::string(v) + c, 8, MPM_H5_F64);
    for (const char* n : {"stress_xx", "stress_yy", "stress_zz", "tau_xy", "tau_yz", "tau_xz",
                          "strain_xx", "strain_yy", "strain_zz", "gamma_xy", "gamma_yz", "gamma_xz"})
      add(n, 8, MPM_H5_F64);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) add("defgrad_" + std::to_string(i) + std::to_string(j), 8, MPM_H5_F64);
    add("initialise_mapping_matrix", 1, MPM_H5_U8);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        add("mapping_matrix_" + std::to_string(i) + std::to_string(j), 8, MPM_H5_F64);
    add("status", 1, MPM_H5_U8);
    add("cell_id", 8, MPM_H5_I64);
    add("material_id", 4, MPM_H5_U32);
    add("nstate_vars", 4, MPM_H5_U32);
    for (int k = 0; k < 20; ++k) add("svars_" + std::to_string(k), 8, MPM_H5_F64);
    for (auto& n : names) cnames.push_back(n.c_str());
  }
};

const RefPod& ref_pod() {
  static const RefPod r;
  return r;
}

}  // namespace

extern "C" {

int mpm_gpu_write_hdf5(mpm_gpu_t h, const char* path) {
  MPM_GUARD(h)
  if (!path) throw InvalidArg("null path");
  const RefPod& L = ref_pod();
  std::vector<uint8_t> rec((size_t)h->np * L.size, 0);
  int64_t n = 0;
  const int rc = mpm_gpu_write_pod(h, rec.data(), h->np, &n, L.size, L.off, L.sz, POD_NFIELDS);
  if (rc != MPM_OK) return rc;
  // H5TBmake_table("Table Title", file, "table", ..., chunk_size 10000, no fill, no compression)
  if (mpm_h5_write_table(path, "Table Title", n, L.size, POD_NFIELDS, L.cnames.data(), L.off, L.type,
                         rec.data(), 10000) != MPM_OK)
    throw InvalidArg(std::string("cannot write ") + path);
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_load_hdf5(mpm_gpu_t h, const char* path) {
  const RefPod& L = ref_pod();
  std::vector<uint8_t> rec;
  int64_t n = 0;
  MPM_GUARD(h)
  if (!path) throw InvalidArg("null path");
  char err[256] = {0};
  if (mpm_h5_read_table(path, &n, L.size, POD_NFIELDS, L.cnames.data(), L.off, L.type, nullptr, 0,
                        err, sizeof(err)) != MPM_OK)
    throw InvalidArg(err);
  rec.assign((size_t)n * L.size, 0);
  if (mpm_h5_read_table(path, &n, L.size, POD_NFIELDS, L.cnames.data(), L.off, L.type, rec.data(), n,
                        err, sizeof(err)) != MPM_OK)
    throw InvalidArg(err);
  MPM_END(h)
  return mpm_gpu_load_pod(h, rec.data(), n, L.size, L.off, L.sz, POD_NFIELDS);
}

}  // extern "C"

// ------------------------------------------------------------ slab decomposition
namespace {

// One x-layer of a tensor-product grid's cells (cell (i, j, k) for fixed i):
// its cell-slot partials (nval values of each of its NV slots, as P2G left
// them) and its particle counts, packed as [ny nz][NV nval] values then
// [ny nz] counts.  T is the partials' element type.
template <typename T>
__global__ void k_halo_pack(const T* partials, const int32_t* cnt, int32_t i, int32_t nx,
                            int64_t ncols, int nvals, T* vals, int32_t* counts) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ncols * nvals) return;
  const int64_t col = e / nvals, v = e % nvals;
  const int64_t c = i + (int64_t)nx * col;
  vals[e] = partials[c * nvals + v];
  if (v == 0) counts[col] = cnt[c];
}
template <typename T>
__global__ void k_halo_unpack(T* partials, int32_t* cnt, int32_t i, int32_t nx, int64_t ncols,
                              int nvals, const T* vals, const int32_t* counts) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ncols * nvals) return;
  const int64_t col = e / nvals, v = e % nvals;
  const int64_t c = i + (int64_t)nx * col;
  partials[c * nvals + v] = vals[e];
  if (v == 0) cnt[c] = counts[col];
}
// particles whose cell's x index is below x_lo or at or above x_hi
__global__ void k_layer_count(const int32_t* cell, int64_t np, int32_t nx, int32_t x_lo, int32_t x_hi,
                              unsigned long long* out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int c = cell[p];
  if (c < 0) return;
  const int i = c % nx;
  if (i < x_lo) atomicAdd(&out[0], 1ull);
  if (i >= x_hi) atomicAdd(&out[1], 1ull);
}

StepArgs slab_step_args(mpm_gpu_t h, int phase) {
  StepArgs a = base_step_args(h);
  set_gravity(h, a, h->step);
  a.phase = phase;
  return a;
}

int64_t halo_cols(mpm_gpu_t h) { return (int64_t)h->gcells[1] * (h->dim == 3 ? h->gcells[2] : 1); }
int halo_nvals(mpm_gpu_t h) { return h->nv * (h->mixed ? mixed_nval(h->dim) : 1 + 3 * h->dim); }

}  // namespace

extern "C" {

int mpm_gpu_step_begin(mpm_gpu_t h) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("initialise or load particles first");
  if (h->cfg.scheme != MPM_SCHEME_USL || h->ntangent > 0 || h->cfg.velocity_update >= MPM_VELOCITY_ASFLIP)
    return fail(h, MPM_ERR_UNSUPPORTED, "the split step follows the USL FLIP / PIC step only");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  refresh_state(h);
  const StepArgs a = slab_step_args(h, 1);
  if (h->mixed)
    launch_step_mixed(h->dim, h->ds, a, h->stream, h->prof);
  else
    launch_step_fp64(h->dim, h->ds, a, h->stream, h->prof);
  ck(cudaGetLastError(), "kernel launch");
  ck(cudaStreamSynchronize(h->stream), "step_begin");
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_step_end(mpm_gpu_t h) {
  MPM_GUARD(h)
  if (!h->initialised) throw InvalidArg("initialise or load particles first");
  if (h->cfg.scheme != MPM_SCHEME_USL || h->ntangent > 0 || h->cfg.velocity_update >= MPM_VELOCITY_ASFLIP)
    return fail(h, MPM_ERR_UNSUPPORTED, "the split step follows the USL FLIP / PIC step only");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const StepArgs a = slab_step_args(h, 2);
  if (h->mixed)
    launch_step_mixed(h->dim, h->ds, a, h->stream, h->prof);
  else
    launch_step_fp64(h->dim, h->ds, a, h->stream, h->prof);
  ck(cudaGetLastError(), "kernel launch");
  ++h->step;
  unsigned words[2] = {0, 0};
  ck(cudaMemcpyAsync(words, h->d_words.p, sizeof(words), cudaMemcpyDeviceToHost, h->stream), "D2H");
  ck(cudaStreamSynchronize(h->stream), "step_end");
  if (words[1] & ERR_NONFINITE) return fail(h, MPM_ERR_NONFINITE, "non-finite particle position");
  if (words[1] & ERR_OUTSIDE) return fail(h, MPM_ERR_OUTSIDE, "Particle(s) outside the mesh domain");
  if (words[1] & ERR_BADCELL) return fail(h, MPM_ERR_INVALID, "corrupt particle cell index");
  if (words[1] & ERR_TIMEOUT) return fail(h, MPM_ERR_TIMEOUT, "a bounded device wait (copy, scan or grid barrier) ran out");
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_halo_bytes(mpm_gpu_t h, int64_t* bytes) {
  MPM_GUARD(h)
  if (!bytes) throw InvalidArg("null bytes");
  if (!h->structured) return fail(h, MPM_ERR_UNSUPPORTED, "halo layers need a tensor-product grid");
  const int64_t cols = halo_cols(h);
  *bytes = cols * halo_nvals(h) * (int64_t)(h->mixed ? sizeof(float) : sizeof(double)) + cols * 4;
  MPM_END(h)
  return MPM_OK;
}

static int halo_copy(mpm_gpu_t h, int32_t layer, void* buf, bool pack) {
  MPM_GUARD(h)
  if (!buf) throw InvalidArg("null halo buffer");
  if (!h->structured) return fail(h, MPM_ERR_UNSUPPORTED, "halo layers need a tensor-product grid");
  if (layer < 0 || layer >= h->gcells[0]) throw InvalidArg("layer outside the grid");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  const int64_t cols = halo_cols(h);
  const int nvals = halo_nvals(h);
  const int64_t n = cols * nvals;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  const size_t esz = h->mixed ? sizeof(float) : sizeof(double);
  int32_t* counts = reinterpret_cast<int32_t*>(static_cast<char*>(buf) + n * esz);
  if (h->mixed) {
    float* v = static_cast<float*>(buf);
    if (pack)
      k_halo_pack<float><<<blocks, 256, 0, h->stream>>>(h->d_partials_f.p, h->d_cnt.p, layer, h->gcells[0],
                                                        cols, nvals, v, counts);
    else
      k_halo_unpack<float><<<blocks, 256, 0, h->stream>>>(h->d_partials_f.p, h->d_cnt.p, layer, h->gcells[0],
                                                          cols, nvals, v, counts);
  } else {
    double* v = static_cast<double*>(buf);
    if (pack)
      k_halo_pack<double><<<blocks, 256, 0, h->stream>>>(h->d_partials.p, h->d_cnt.p, layer, h->gcells[0],
                                                         cols, nvals, v, counts);
    else
      k_halo_unpack<double><<<blocks, 256, 0, h->stream>>>(h->d_partials.p, h->d_cnt.p, layer,
                                                           h->gcells[0], cols, nvals, v, counts);
  }
  ck(cudaGetLastError(), "halo kernel");
  ck(cudaStreamSynchronize(h->stream), "halo");
  MPM_END(h)
  return MPM_OK;
}

int mpm_gpu_halo_pack(mpm_gpu_t h, int32_t layer, void* dst) { return halo_copy(h, layer, dst, true); }
int mpm_gpu_halo_unpack(mpm_gpu_t h, int32_t layer, const void* src) {
  return halo_copy(h, layer, const_cast<void*>(src), false);
}

int mpm_gpu_layer_count(mpm_gpu_t h, int32_t x_lo, int32_t x_hi, int64_t* below, int64_t* above) {
  MPM_GUARD(h)
  if (!below || !above) throw InvalidArg("null output");
  if (!h->structured) return fail(h, MPM_ERR_UNSUPPORTED, "layers need a tensor-product grid");
  ck(cudaSetDevice(h->cfg.device), "cudaSetDevice");
  DevBuf<unsigned long long> c;
  c.alloc(2);
  ck(cudaMemsetAsync(c.p, 0, 16, h->stream), "memset");
  if (h->npad > 0)
    k_layer_count<<<(unsigned)((h->npad + 255) / 256), 256, 0, h->stream>>>(h->d_cell.p, h->npad,
                                                                           h->gcells[0], x_lo, x_hi, c.p);
  unsigned long long r[2] = {0, 0};
  c.download(r, 2, h->stream);
  ck(cudaStreamSynchronize(h->stream), "layer count");
  *below = (int64_t)r[0];
  *above = (int64_t)r[1];
  MPM_END(h)
  return MPM_OK;
}

}  // extern "C"
