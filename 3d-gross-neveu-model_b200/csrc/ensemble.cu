// ensemble.cu -- host side of the batched chains (ensemble_kernel.cuh) and
// their extern "C" functions (gn_ensemble_* in include/gn_b200.h).
//
// One trajectory of every chain is a fixed sequence of launches: a memset of
// the launches' work queues and team barriers, then one persistent cooperative
// kernel per slice of the op list (the refresh and initial solve, one MD step
// each, the last step with the energy and the Metropolis test).  The sequence
// is captured once as a CUDA graph and replayed per trajectory.  The team
// layout (blocks per group for the big chains, and which chains are big) is
// chosen by tune(): it times the refresh-and-solve slice, which has no effect
// on any chain's results, for every candidate layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <vector>

#include "../../include/gn_b200.h"
#define GN_DEFINE_ENSEMBLE_KERNEL
#include "ensemble_kernel.cuh"
#include "trace.h"
#include "checkpoint.h"
#include "errors.h"
#include "launch.h"
#include "schedule.h"

namespace gn {

constexpr double kEnsDelta = 0.01;  // reliable update when |r^| drops by this factor (as mixed.cu)
constexpr int kEnsReliableEvery = 100;

class Ensemble {
 public:
  Ensemble(int n, const int *L, const double *beta_s, const unsigned long long *ids, unsigned long long seed,
           int device);
  ~Ensemble();
  int n() const { return n_; }
  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  void load_sigma(int c, const double *h);
  void store_sigma(int c, double *sigma, double *sm);
  void set_layout(int gs, long long big_min);
  void set_precision(int prec);
  void tune(const gn_ens_params &p, int *gs, long long *big_min);
  void run(const gn_ens_params &p, int ntraj, bool graph);
  void stats(gn_chain_stats *out, bool reset);
  void observables(double *out);
  int checkpoint_save(int c, const char *path, const char *copy, const gn_hmc_counters *cnt);
  void set_autoregulation(int c, bool on);
  EnsState state(int c);
  void set_state(int c, const EnsState &h);
  int checkpoint_load(int c, const char *path, const char *copy, gn_hmc_counters *cnt);
  void info(int *gs, long long *big_min, int *graph_used, int *launches);

 private:
  void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw GnError(GN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  struct Plan {  // the op list of a trajectory and its slices
    std::vector<EnsOp> ops;
    std::vector<int> node_begin;  // node k runs ops [node_begin[k], node_begin[k + 1])
    EnsOp *d_ops = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool graph_failed = false;
    int layout_epoch = -1;  // the layout the graph was captured with
  };
  Plan &plan_for(const gn_ens_params &p);
  void build_order();
  void launch_node(const Plan &pl, int k, double tol);
  void enqueue_trajectory(const Plan &pl, double tol);
  void check_err();

  int device_ = 0, n_ = 0, capacity_ = 0;
  cudaStream_t stream_ = nullptr;
  unsigned long long seed_ = 0;
  std::vector<EnsChain> chains_;
  void *arena_ = nullptr;
  EnsChain *d_chains_ = nullptr;
  EnsState *d_states_ = nullptr;
  int *d_order_ = nullptr;
  int *d_queue_ = nullptr;      // [kMaxNodes][kMaxTiers]
  PhaseBar *d_bars_ = nullptr;  // [kMaxNodes][kMaxTiers][capacity]
  double *d_partials_ = nullptr;
  CgState *d_cg_state_ = nullptr;
  int *d_err_ = nullptr;
  int gs_ = 1;
  long long big_min_ = 0;
  int nbig_ = 0;
  int layout_epoch_ = 0;
  bool last_graph_ = false;
  int last_launches_ = 0;
  std::map<std::vector<double>, std::unique_ptr<Plan>> plans_;
  static constexpr int kMaxNodes = 64;
};

static size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

Ensemble::Ensemble(int n, const int *L, const double *beta_s, const unsigned long long *ids, unsigned long long seed,
                   int device)
    : device_(device), n_(n), seed_(seed) {
  if (n < 1) throw GnError(GN_ERR_ARG, "an ensemble needs at least one chain");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw GnError(GN_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) throw GnError(GN_ERR_ARG, "no such device");
  check(cudaSetDevice(device), "cudaSetDevice");
  cudaDeviceProp prop;
  check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major != 10) throw GnError(GN_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only");
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  capacity_ = coop_capacity((const void *)ens_node_kernel, kEnsThreads);
  if (capacity_ < 1) throw GnError(GN_ERR_CUDA, "the batched kernel cannot be resident as a cooperative grid");
  // ---- one arena for every chain's arrays; a two-plane array is one block of
  // 2V values (plane f at f V), every array starts on a 256-byte boundary
  auto carve = [&](char *base, int c, EnsChain *ch) -> size_t {
    const size_t V = size_t(L[c]) * L[c] * L[c];
    size_t used = 0;
    auto dv = [&](int planes) {
      double *q = reinterpret_cast<double *>(base + used);
      used += round256(planes * V * sizeof(double));
      return q;
    };
    auto fv = [&](int planes) {
      float *q = reinterpret_cast<float *>(base + used);
      used += round256(planes * V * sizeof(float));
      return q;
    };
    double *s0 = dv(1), *s1 = dv(1), *sm = dv(1), *P = dv(1), *F = dv(1), *save = dv(1);
    double *chi = dv(2), *phi = dv(2), *X = dv(2), *Y = dv(2), *t64 = dv(2);
    double *r64 = dv(2), *pa64 = dv(2), *pb64 = dv(2);
    float *sm32 = fv(1), *rh = fv(2), *ph = fv(2), *uh = fv(2), *ah = fv(2), *xh = fv(2);
    if (ch) {
      ch->g = make_geom(L[c]);
      ch->w = row_width(L[c], 4);
      ch->beta_s = beta_s[c];
      ch->stream = ids ? ids[c] : (unsigned long long)c;
      ch->sigma[0] = s0;
      ch->sigma[1] = s1;
      ch->sm = sm;
      ch->P = P;
      ch->F = F;
      ch->sigma_save = save;
      ch->chi = chi;
      ch->phi = phi;
      ch->X = X;
      ch->Y = Y;
      ch->t64 = t64;
      ch->sm32 = sm32;
      ch->rh = rh;
      ch->ph = ph;
      ch->uh = uh;
      ch->ah = ah;
      ch->xh = xh;
      ch->r64 = r64;
      ch->pa64 = pa64;
      ch->pb64 = pb64;
      ch->precision = GN_PREC_MIXED;
    }
    return used;
  };
  size_t total = 0;
  std::vector<size_t> off(n);
  for (int c = 0; c < n; c++) {
    if (L[c] < 4 || L[c] > 256 || (L[c] & 1)) throw GnError(GN_ERR_ARG, "every L must be even and in [4, 256]");
    off[c] = total;
    total += carve(nullptr, c, nullptr);
  }
  check(cudaMalloc(&arena_, total), "cudaMalloc ensemble arena");
  check(cudaMemsetAsync(arena_, 0, total, stream_), "memset arena");
  chains_.resize(n);
  for (int c = 0; c < n; c++) carve(static_cast<char *>(arena_) + off[c], c, &chains_[c]);
  check(cudaMalloc(&d_states_, n * sizeof(EnsState)), "cudaMalloc states");
  for (int c = 0; c < n; c++) {
    chains_[c].state = d_states_ + c;
    chains_[c].op_begin = chains_[c].op_end = 0;
  }
  check(cudaMalloc(&d_chains_, n * sizeof(EnsChain)), "cudaMalloc chains");
  check(cudaMemcpyAsync(d_chains_, chains_.data(), n * sizeof(EnsChain), cudaMemcpyHostToDevice, stream_), "copy");
  check(cudaMemsetAsync(d_states_, 0, n * sizeof(EnsState), stream_), "memset states");
  check(cudaMalloc(&d_order_, n * sizeof(int)), "cudaMalloc order");
  check(cudaMalloc(&d_queue_, kMaxNodes * kMaxTiers * sizeof(int)), "cudaMalloc queue");
  check(cudaMalloc(&d_bars_, size_t(kMaxNodes) * kMaxTiers * capacity_ * sizeof(PhaseBar)), "cudaMalloc bars");
  // two regions: the teams' partial sums, and those of the second flavour of two-team solves
  check(cudaMalloc(&d_partials_, size_t(2) * kMaxTiers * capacity_ * 2 * (kSyncQ + 1) * sizeof(double)),
        "cudaMalloc partials");
  check(cudaMalloc(&d_cg_state_, size_t(capacity_) * kMaxRhs * sizeof(CgState)), "cudaMalloc cg state");
  check(cudaMalloc(&d_err_, sizeof(int)), "cudaMalloc err");
  check(cudaMemsetAsync(d_err_, 0, sizeof(int), stream_), "memset err");
  set_layout(1, 0);
  check(cudaStreamSynchronize(stream_), "ensemble set-up");
}

Ensemble::~Ensemble() {
  cudaSetDevice(device_);
  cudaStreamSynchronize(stream_);
  for (auto &kv : plans_) {
    if (kv.second->graph) cudaGraphExecDestroy(kv.second->graph);
    if (kv.second->d_ops) cudaFree(kv.second->d_ops);
  }
  cudaFree(arena_);
  cudaFree(d_chains_);
  cudaFree(d_states_);
  cudaFree(d_order_);
  cudaFree(d_queue_);
  cudaFree(d_bars_);
  cudaFree(d_partials_);
  cudaFree(d_cg_state_);
  cudaFree(d_err_);
  cudaStreamDestroy(stream_);
}

void Ensemble::load_sigma(int c, const double *h) {
  if (c < 0 || c >= n_ || h == nullptr) throw GnError(GN_ERR_ARG, "bad chain or null sigma");
  const EnsChain &ch = chains_[c];
  const size_t V = size_t(ch.g.V);
  int cur = 0;
  check(cudaMemcpyAsync(&cur, &d_states_[c].cur, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "sync");
  check(cudaMemcpyAsync(ch.sigma[cur], h, V * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload sigma");
  sigma_mass_kernel<double><<<unsigned((V + kOpThreads - 1) / kOpThreads), kOpThreads, 0, stream_>>>(
      ch.g, ch.sigma[cur], nullptr, 0.0, nullptr, ch.sm);
  check(cudaGetLastError(), "sigma_mass_kernel");
  check(cudaStreamSynchronize(stream_), "load sigma");
}

void Ensemble::store_sigma(int c, double *sigma, double *sm) {
  if (c < 0 || c >= n_) throw GnError(GN_ERR_ARG, "bad chain");
  const EnsChain &ch = chains_[c];
  const size_t V = size_t(ch.g.V);
  int cur = 0;
  check(cudaMemcpyAsync(&cur, &d_states_[c].cur, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "sync");
  if (sigma) check(cudaMemcpyAsync(sigma, ch.sigma[cur], V * sizeof(double), cudaMemcpyDeviceToHost, stream_), "copy");
  if (sm) check(cudaMemcpyAsync(sm, ch.sm, V * sizeof(double), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "store sigma");
}

// Chains by decreasing volume (ties by index); the big ones (V >= big_min,
// with groups of more than one block) first.
void Ensemble::build_order() {
  std::vector<int> order(n_);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return chains_[a].g.V > chains_[b].g.V; });
  nbig_ = 0;
  if (gs_ > 1)
    for (int c : order)
      if (chains_[c].g.V >= big_min_) nbig_++;
  check(cudaMemcpyAsync(d_order_, order.data(), n_ * sizeof(int), cudaMemcpyHostToDevice, stream_), "copy order");
  check(cudaStreamSynchronize(stream_), "order");
}

// The chains' solver precision (uploaded with the chain table when it changes).
void Ensemble::set_precision(int prec) {
  if (!chains_.empty() && chains_[0].precision == prec) return;
  for (EnsChain &ch : chains_) ch.precision = prec;
  check(cudaMemcpyAsync(d_chains_, chains_.data(), n_ * sizeof(EnsChain), cudaMemcpyHostToDevice, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "precision");
}

void Ensemble::set_layout(int gs, long long big_min) {
  if (gs < 1 || gs > capacity_) throw GnError(GN_ERR_ARG, "blocks per group out of range");
  gs_ = gs;
  big_min_ = big_min;
  build_order();
  layout_epoch_++;
}

Ensemble::Plan &Ensemble::plan_for(const gn_ens_params &p) {
  const std::vector<double> key = {p.eps, double(p.steps), double(p.integrator), p.tol, double(p.precision)};
  auto it = plans_.find(key);
  if (it != plans_.end()) return *it->second;
  auto pl = std::make_unique<Plan>();
  // translation of the integrator's op list (schedule.h): a force and the
  // momentum step after it are one E_FORCE; every force is a solve first
  std::vector<EnsOp> body;
  const std::vector<Op> ops = schedule(p.integrator, p.eps, p.steps);
  for (size_t k = 0; k < ops.size(); k++) {
    const Op &o = ops[k];
    if (o.op == OP_F_MED || o.op == OP_F_HIGH) {
      body.push_back({E_SOLVE, 0.0});
      double c = 0.0;
      if (k + 1 < ops.size() && ops[k + 1].op == OP_P) {
        c = ops[k + 1].c;
        k++;
      }
      body.push_back({E_FORCE, c});
    } else if (o.op == OP_P) {
      body.push_back({E_P, o.c});
    } else if (o.op == OP_Q) {
      body.push_back({E_Q, o.c});
    } else {
      body.push_back({E_SOLVE, 0.0});
    }
  }
  // slices: the refresh with the initial solve and H0, then one MD step per
  // launch (two solves for the two-force integrators), the energy and the
  // Metropolis test in the last one
  pl->ops = {{E_REFRESH, 0.0}, {E_PHI, 0.0}, {E_SOLVE, 0.0}, {E_ENERGY0, 0.0}};
  pl->node_begin.push_back(0);
  const int per_node = (p.integrator == GN_LF2) ? 1 : 2;
  int solves = per_node;  // a new slice at the first solve
  for (const EnsOp &o : body) {
    if (o.code == E_SOLVE) {
      if (solves == per_node) {
        pl->node_begin.push_back(int(pl->ops.size()));
        solves = 0;
      }
      solves++;
    }
    pl->ops.push_back(o);
  }
  pl->ops.push_back({E_ENERGY1, 0.0});
  pl->ops.push_back({E_METROPOLIS, 0.0});
  pl->node_begin.push_back(int(pl->ops.size()));
  if (int(pl->node_begin.size()) - 1 > kMaxNodes) throw GnError(GN_ERR_ARG, "too many MD steps for one trajectory");
  check(cudaMalloc(&pl->d_ops, pl->ops.size() * sizeof(EnsOp)), "cudaMalloc ops");
  check(cudaMemcpyAsync(pl->d_ops, pl->ops.data(), pl->ops.size() * sizeof(EnsOp), cudaMemcpyHostToDevice, stream_),
        "copy ops");
  check(cudaStreamSynchronize(stream_), "ops");
  Plan &ref = *pl;
  plans_[key] = std::move(pl);
  return ref;
}

void Ensemble::launch_node(const Plan &pl, int k, double tol) {
  EnsLaunch a;
  a.chains = d_chains_;
  a.nchains = n_;
  a.order = d_order_;
  if (gs_ > 1 && nbig_ > 0) {  // the big chains on teams of gs_ blocks, the rest on single blocks
    a.ntier = 2;
    a.tier_gs[0] = gs_;
    a.tier_end[0] = nbig_;
    a.tier_gs[1] = 1;
    a.tier_end[1] = n_;
  } else {
    a.ntier = 1;
    a.tier_gs[0] = 1;
    a.tier_end[0] = n_;
  }
  a.ops = pl.d_ops;
  a.op_begin = pl.node_begin[k];
  a.op_end = pl.node_begin[k + 1];
  a.queue = d_queue_ + kMaxTiers * k;
  a.bars = d_bars_ + size_t(k) * kMaxTiers * capacity_;
  a.partials = d_partials_;
  a.partials2 = d_partials_ + size_t(kMaxTiers) * capacity_ * 2 * (kSyncQ + 1);
  a.duo = ens_duo_enabled();
  a.cg_state = d_cg_state_;
  a.err = d_err_;
  a.seed = seed_;
  a.tol = tol;
  a.delta = kEnsDelta;
  a.n_ru = kEnsReliableEvery;
  void *args[] = {(void *)&a};
  check(cudaLaunchCooperativeKernel((const void *)ens_node_kernel, dim3(capacity_), dim3(kEnsThreads), args, 0,
                                    stream_),
        "ens_node_kernel launch");
}

// One trajectory of every chain: zero the slices' queues and barriers, then the slices.
void Ensemble::enqueue_trajectory(const Plan &pl, double tol) {
  const int nodes = int(pl.node_begin.size()) - 1;
  check(cudaMemsetAsync(d_queue_, 0, size_t(nodes) * kMaxTiers * sizeof(int), stream_), "memset queue");
  check(cudaMemsetAsync(d_bars_, 0, size_t(nodes) * kMaxTiers * capacity_ * sizeof(PhaseBar), stream_),
        "memset bars");
  for (int k = 0; k < nodes; k++) launch_node(pl, k, tol);
}

void Ensemble::check_err() {
  int h = 0;
  check(cudaMemcpyAsync(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy err");
  check(cudaStreamSynchronize(stream_), "ensemble sync");
  if (h != 0) {
    cudaMemsetAsync(d_err_, 0, sizeof(int), stream_);
    cudaStreamSynchronize(stream_);
    throw GnError(GN_ERR_TIMEOUT, "batched kernel: a team barrier timed out");
  }
}

void Ensemble::run(const gn_ens_params &p, int ntraj, bool graph) {
  TraceRange tr("gn ensemble run");
  if (p.steps < 1 || p.integrator < 0 || p.integrator > 2 || !(p.tol > 0.0) || ntraj < 0)
    throw GnError(GN_ERR_ARG, "bad ensemble parameters");
  if (p.precision != GN_PREC_MIXED && p.precision != GN_PREC_FP64)
    throw GnError(GN_ERR_ARG, "ensemble precision: GN_PREC_MIXED or GN_PREC_FP64");
  set_precision(p.precision);
  Plan &pl = plan_for(p);
  last_launches_ = int(pl.node_begin.size()) - 1;
  if (graph && !pl.graph_failed && (pl.graph == nullptr || pl.layout_epoch != layout_epoch_)) {
    if (pl.graph) {
      cudaGraphExecDestroy(pl.graph);
      pl.graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    bool okc = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (okc) {
      try {
        enqueue_trajectory(pl, p.tol);
      } catch (const GnError &) {
        okc = false;
      }
      okc = (cudaStreamEndCapture(stream_, &g) == cudaSuccess) && okc;
    }
    if (okc && g) okc = cudaGraphInstantiate(&pl.graph, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (!okc) {
      pl.graph = nullptr;
      pl.graph_failed = true;
    }
    pl.layout_epoch = layout_epoch_;
  }
  last_graph_ = graph && pl.graph != nullptr;
  for (int t = 0; t < ntraj; t++) {
    if (last_graph_) check(cudaGraphLaunch(pl.graph, stream_), "cudaGraphLaunch");
    else enqueue_trajectory(pl, p.tol);
  }
  check_err();
}

void Ensemble::tune(const gn_ens_params &p, int *gs_out, long long *big_out) {
  set_precision(p.precision == GN_PREC_FP64 ? GN_PREC_FP64 : GN_PREC_MIXED);
  Plan &pl = plan_for(p);
  std::vector<long long> vols;
  for (const EnsChain &ch : chains_) vols.push_back(ch.g.V);
  std::sort(vols.begin(), vols.end());
  vols.erase(std::unique(vols.begin(), vols.end()), vols.end());
  std::vector<std::pair<int, long long>> cand = {{1, 0}};
  for (int gs : {2, 4, 8, 16})
    if (gs <= capacity_)
      for (long long v : vols) cand.push_back({gs, v});
  cudaEvent_t e0, e1;
  check(cudaEventCreate(&e0), "event");
  check(cudaEventCreate(&e1), "event");
  float best = 1e30f;
  std::pair<int, long long> pick = cand[0];
  for (const auto &cd : cand) {
    set_layout(cd.first, cd.second);
    float ms = 0.f;
    for (int rep = 0; rep < 2; rep++) {  // the first launch warms up; the second is timed
      check(cudaMemsetAsync(d_queue_, 0, kMaxTiers * sizeof(int), stream_), "memset queue");
      check(cudaMemsetAsync(d_bars_, 0, size_t(kMaxTiers) * capacity_ * sizeof(PhaseBar), stream_), "memset bars");
      check(cudaEventRecord(e0, stream_), "record");
      launch_node(pl, 0, p.tol);
      check(cudaEventRecord(e1, stream_), "record");
      check_err();
      check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    }
    if (ms < best) {
      best = ms;
      pick = cd;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  set_layout(pick.first, pick.second);
  if (gs_out) *gs_out = gs_;
  if (big_out) *big_out = big_min_;
}

void Ensemble::stats(gn_chain_stats *out, bool reset) {
  std::vector<EnsState> h(n_);
  check(cudaMemcpyAsync(h.data(), d_states_, n_ * sizeof(EnsState), cudaMemcpyDeviceToHost, stream_), "copy states");
  check(cudaStreamSynchronize(stream_), "states");
  for (int c = 0; c < n_; c++) {
    if (out) {
      gn_chain_stats &o = out[c];
      o.trajectories = h[c].n;
      o.accepted = h[c].nacc;
      o.failed = h[c].fails;
      o.cg_iterations = h[c].iters;
      o.reliable_updates = h[c].reliable;
      o.sum_dH = h[c].sum_dH;
      o.sum_exp_mdH = h[c].sum_exp_mdH;
      o.sum_sigma2 = h[c].sum_sigma2;
      o.last_dH = h[c].last_dH;
      o.last_accepted = h[c].last_acc;
      o.total_trajectories = h[c].ntraj;
      o.total_accepted = h[c].total_acc;
      o.story = h[c].story;
      o.local_accepted = h[c].local_acc;
      o.local_done = h[c].local_done;
      o.epsilon_scale = h[c].eps_scale > 0.0 ? h[c].eps_scale : 1.0;
    }
    if (reset) {
      h[c].n = h[c].nacc = h[c].iters = h[c].reliable = h[c].fails = 0;
      h[c].sum_dH = h[c].sum_exp_mdH = h[c].sum_sigma2 = 0.0;
      for (int q = 0; q < kSigmaObs; q++) h[c].sum_obs[q] = 0.0;
    }
  }
  if (reset) {
    check(cudaMemcpyAsync(d_states_, h.data(), n_ * sizeof(EnsState), cudaMemcpyHostToDevice, stream_), "copy");
    check(cudaStreamSynchronize(stream_), "states");
  }
}

void Ensemble::observables(double *out) {
  std::vector<EnsState> h(n_);
  check(cudaMemcpyAsync(h.data(), d_states_, n_ * sizeof(EnsState), cudaMemcpyDeviceToHost, stream_), "copy states");
  check(cudaStreamSynchronize(stream_), "states");
  for (int c = 0; c < n_; c++)
    for (int q = 0; q < kSigmaObs; q++)
      out[size_t(c) * kSigmaObs + q] = h[c].n > 0 ? h[c].sum_obs[q] / double(h[c].n) : 0.0;
}

EnsState Ensemble::state(int c) {
  EnsState h;
  check(cudaMemcpyAsync(&h, d_states_ + c, sizeof(EnsState), cudaMemcpyDeviceToHost, stream_), "copy state");
  check(cudaStreamSynchronize(stream_), "state");
  return h;
}

void Ensemble::set_state(int c, const EnsState &h) {
  check(cudaMemcpyAsync(d_states_ + c, &h, sizeof(EnsState), cudaMemcpyHostToDevice, stream_), "copy state");
  check(cudaStreamSynchronize(stream_), "state");
}

void Ensemble::set_autoregulation(int c, bool on) {
  if (c >= n_) throw GnError(GN_ERR_ARG, "bad chain");
  for (int k = (c < 0 ? 0 : c); k < (c < 0 ? n_ : c + 1); k++) {
    EnsState h = state(k);
    h.autoreg = on ? 1 : 0;
    h.local_acc = h.local_done = 0;
    set_state(k, h);
  }
}

int Ensemble::checkpoint_save(int c, const char *path, const char *copy, const gn_hmc_counters *cnt) {
  if (c < 0 || c >= n_) throw GnError(GN_ERR_ARG, "bad chain");
  const size_t V = size_t(chains_[c].g.V);
  std::vector<double> sigma(V), sm(V);
  store_sigma(c, sigma.data(), sm.data());
  gn_hmc_counters own;
  memset(&own, 0, sizeof own);
  if (cnt == nullptr) {  // the chain's own bookkeeping
    const EnsState h = state(c);
    own.accepted_sigma = int(h.total_acc);
    own.done_sigma = int(h.ntraj);
    own.story_sigma = h.story;
    cnt = &own;
  }
  return write_lattice_file(path, copy, chains_[c].g.L, sigma.data(), sm.data(), nullptr, *cnt);
}

int Ensemble::checkpoint_load(int c, const char *path, const char *copy, gn_hmc_counters *cnt) {
  if (c < 0 || c >= n_) throw GnError(GN_ERR_ARG, "bad chain");
  const size_t V = size_t(chains_[c].g.V);
  std::vector<double> old(V);
  store_sigma(c, old.data(), nullptr);
  bool replaced = false;
  auto sm_of = [&](const double *sigma, double *sm) {  // the chain's own arrays; restored on failure
    load_sigma(c, sigma);
    store_sigma(c, nullptr, sm);
    replaced = true;
  };
  auto accept = [&](const double *sigma) { load_sigma(c, sigma); };
  gn_hmc_counters got;
  const int st = load_lattice(path, copy, chains_[c].g.L, &got, sm_of, accept);
  if (st != GN_OK) {
    if (replaced) load_sigma(c, old.data());
    return st;
  }
  EnsState h = state(c);  // resume the chain's bookkeeping and Philox counter
  h.ntraj = got.done_sigma;
  h.total_acc = got.accepted_sigma;
  h.story = got.story_sigma;
  set_state(c, h);
  if (cnt) *cnt = got;
  return GN_OK;
}

void Ensemble::info(int *gs, long long *big_min, int *graph_used, int *launches) {
  if (gs) *gs = gs_;
  if (big_min) *big_min = big_min_;
  if (graph_used) *graph_used = last_graph_ ? 1 : 0;
  if (launches) *launches = last_launches_;
}

}  // namespace gn

struct gn_ensemble {
  std::unique_ptr<gn::Ensemble> e;
};

namespace {

template <typename F>
int ens_guarded(gn_ensemble *e, F &&f) {
  if (e == nullptr || !e->e) return gn::set_last_error(GN_ERR_ARG, "null ensemble");
  try {
    cudaSetDevice(e->e->device());
    return f(*e->e);
  } catch (const gn::GnError &x) {
    return gn::set_last_error(x.status, x.what());
  } catch (const std::exception &x) {
    return gn::set_last_error(GN_ERR_CUDA, x.what());
  }
}

}  // namespace

extern "C" {

int gn_ensemble_create(gn_ensemble **out, int nchains, const int *L, const double *beta_s,
                       const unsigned long long *stream_ids, unsigned long long seed, int device) {
  if (out == nullptr || L == nullptr || beta_s == nullptr) return gn::set_last_error(GN_ERR_ARG, "null argument");
  *out = nullptr;
  try {
    auto e = std::make_unique<gn_ensemble>();
    e->e = std::make_unique<gn::Ensemble>(nchains, L, beta_s, stream_ids, seed, device);
    *out = e.release();
    return GN_OK;
  } catch (const gn::GnError &x) {
    return gn::set_last_error(x.status, x.what());
  } catch (const std::exception &x) {
    return gn::set_last_error(GN_ERR_CUDA, x.what());
  }
}

void gn_ensemble_destroy(gn_ensemble *e) { delete e; }

void *gn_ensemble_stream(gn_ensemble *e) { return (e && e->e) ? (void *)e->e->stream() : nullptr; }

int gn_ensemble_load_sigma(gn_ensemble *e, int chain, const double *sigma) {
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.load_sigma(chain, sigma);
    return GN_OK;
  });
}

int gn_ensemble_store_sigma(gn_ensemble *e, int chain, double *sigma, double *sigmamass) {
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.store_sigma(chain, sigma, sigmamass);
    return GN_OK;
  });
}

int gn_ensemble_set_layout(gn_ensemble *e, int group_blocks, long long big_min_volume) {
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.set_layout(group_blocks, big_min_volume);
    return GN_OK;
  });
}

int gn_ensemble_tune(gn_ensemble *e, const gn_ens_params *p, int *group_blocks, long long *big_min_volume) {
  if (p == nullptr) return gn::set_last_error(GN_ERR_ARG, "null parameters");
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.tune(*p, group_blocks, big_min_volume);
    return GN_OK;
  });
}

int gn_ensemble_run(gn_ensemble *e, const gn_ens_params *p, int ntraj, int use_graph) {
  if (p == nullptr) return gn::set_last_error(GN_ERR_ARG, "null parameters");
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.run(*p, ntraj, use_graph != 0);
    return GN_OK;
  });
}

int gn_ensemble_stats(gn_ensemble *e, gn_chain_stats *out, int reset) {
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.stats(out, reset != 0);
    return GN_OK;
  });
}

int gn_ensemble_observables(gn_ensemble *e, double *out) {
  if (out == nullptr) return gn::set_last_error(GN_ERR_ARG, "null pointer");
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.observables(out);
    return GN_OK;
  });
}

int gn_ensemble_set_autoregulation(gn_ensemble *e, int chain, int on) {
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.set_autoregulation(chain, on != 0);
    return GN_OK;
  });
}

int gn_ensemble_checkpoint_save(gn_ensemble *e, int chain, const char *path, const char *path_copy,
                                const gn_hmc_counters *c) {
  if (path == nullptr) return gn::set_last_error(GN_ERR_ARG, "null pointer");
  return ens_guarded(e, [&](gn::Ensemble &E) -> int {
    const int st = E.checkpoint_save(chain, path, path_copy, c);
    return st == GN_OK ? GN_OK : gn::set_last_error(st, "cannot write the lattice file");
  });
}

int gn_ensemble_checkpoint_load(gn_ensemble *e, int chain, const char *path, const char *path_copy,
                                gn_hmc_counters *c) {
  if (path == nullptr) return gn::set_last_error(GN_ERR_ARG, "null pointer");
  return ens_guarded(e, [&](gn::Ensemble &E) -> int {
    const int st = E.checkpoint_load(chain, path, path_copy, c);
    if (st == GN_ERR_NOT_FOUND) return gn::set_last_error(st, "no lattice file (a fresh start)");
    if (st != GN_OK) return gn::set_last_error(st, "no lattice file passed its check");
    return GN_OK;
  });
}

int gn_ensemble_info(gn_ensemble *e, int *group_blocks, long long *big_min_volume, int *graph_used,
                     int *launches_per_trajectory) {
  return ens_guarded(e, [&](gn::Ensemble &E) {
    E.info(group_blocks, big_min_volume, graph_used, launches_per_trajectory);
    return GN_OK;
  });
}

}  // extern "C"
