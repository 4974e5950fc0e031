// serve.cu -- a request server over resident chains with continuous batching
// (gn_server_* in include/gn_b200.h).
//
// Chains keep sigma (two ping-pong buffers) and its mass resident between
// requests.  A request -- one HMC trajectory of a chain, one solve of
// (M M^T) x = b with b ~ N(0, 1) at the chain's sigma, or a condensate
// estimate from Z2 noise vectors -- is a program of slices of the batched
// kernel's ops (ensemble_kernel.cuh).  Every step launches the batched kernel
// once for all running requests, each advancing by its next slice (requests
// of different kinds and lattice sizes share the launch), then retires the
// finished ones and admits queued ones: in arrival order, when the request's
// chain is free and its work arrays fit the memory budget.  Work arrays come
// from the stream-ordered allocator at admission and go back at retirement.
// A request's numbers depend only on its chain's state and its serial number on
// that chain (the Philox counter of its draws), not on the requests beside it --
// bit for bit where its team size is fixed; the top tier's team size follows
// the load (a lone big request gets the whole GPU), which changes only the
// order of the solver's sums.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <numeric>
#include <vector>

#include "../../include/gn_b200.h"
#include "trace.h"
#include "ensemble_kernel.cuh"  // declares ens_node_kernel (defined in ensemble.cu)
#include "errors.h"
#include "launch.h"
#include "schedule.h"

namespace gn {

constexpr int kMaxNoise = 64;  // Z2 vectors of one condensate request

class Server {
 public:
  Server(const gn_ens_params &traj, size_t budget, unsigned long long seed, int ntier, const int *tier_blocks,
         const long long *tier_min_volume, int device);
  ~Server();
  int device() const { return device_; }
  int add_chain(int L, double beta, const double *sigma, unsigned long long stream_id);
  double clock() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }
  long long submit(int chain, int type, int nnoise, double t_arrival);
  int step();
  void request(long long id, gn_request_info *out);
  void solution(long long id, double *x);
  void chain_sigma(int chain, double *sigma);
  void load(int *running, int *queued, long long *bytes);

 private:
  struct Chain {
    int L;
    Geom g;
    int w;
    double beta;
    unsigned long long stream;
    double *sigma[2] = {nullptr, nullptr};
    double *sm = nullptr;
    bool busy = false;
    unsigned long long nreq = 0;  // requests submitted to the chain: the next one's serial number
  };
  struct Program {  // slices [node_begin[k], node_begin[k + 1]) of the op array
    std::vector<int> node_begin;
    std::vector<int> solves;  // solves in slice k
  };
  struct Req {
    gn_request_info info;
    int nslices = 0, next = 0, take = 1;  // slices done; slices this step
    const Program *prog = nullptr;
    long long iters0 = 0;       // the chain's solver iteration count at admission
    unsigned long long serial;  // the request's number on its chain: the Philox counter of its draws
    void *work = nullptr;
    size_t bytes = 0;
    std::vector<double> x;  // a finished solve's solution
  };
  void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw GnError(GN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  static size_t work_bytes(size_t V);
  EnsChain chain_entry(const Req &r);
  static double *work_X(const Req &r, size_t V);
  void admit();

  int device_ = 0, capacity_ = 0;
  std::vector<int> tier_gs_;          // team sizes, decreasing; the last tier (single blocks) is implicit
  std::vector<long long> tier_min_;   // a chain with V >= tier_min_[t] (and below the earlier tiers) runs in tier t
  int tier_of(long long V) const {
    for (size_t t = 0; t < tier_min_.size(); t++)
      if (V >= tier_min_[t]) return int(t);
    return int(tier_gs_.size());
  }
  size_t budget_ = 0, in_use_ = 0;
  unsigned long long seed_ = 0;
  double tol_ = 1e-10;
  int precision_ = GN_PREC_MIXED;
  cudaStream_t stream_ = nullptr;
  // the requests' work arrays come from a pool of the server's own that keeps
  // its memory mapped up to the budget: the device's default pool returns
  // freed memory at every synchronisation, and mapping it again on the next
  // admission took up to 0.8 s on B200, stalling every request behind it
  cudaMemPool_t pool_ = nullptr;
  std::chrono::steady_clock::time_point t0_;
  std::vector<Chain> chains_;
  EnsState *d_states_ = nullptr;  // [kMaxChains]
  static constexpr int kMaxChains = 4096;
  std::vector<EnsOp> ops_;
  EnsOp *d_ops_ = nullptr;
  Program traj_, solve_, cond_;
  std::deque<long long> queue_;
  std::vector<long long> running_;
  std::map<long long, Req> reqs_;
  long long next_id_ = 0;
  EnsChain *d_table_ = nullptr, *h_table_ = nullptr;
  int *d_order_ = nullptr;
  int *d_queue_ = nullptr;
  PhaseBar *d_bars_ = nullptr;
  double *d_partials_ = nullptr;
  CgState *d_cg_state_ = nullptr;
  int *d_err_ = nullptr;
  EnsState *h_states_ = nullptr;
};

static size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// A running request's arrays: P, F, sigma_save (1 plane each), chi, phi, X,
// Y, t64 (2 planes), sm32 (1 plane of float), the mixed solver's r^, p^, u^,
// a^, x^ (2 planes of float each), the FP64 solver's r, p, p' (2 planes each).
size_t Server::work_bytes(size_t V) {
  return 3 * round256(V * 8) + 5 * round256(2 * V * 8) + round256(V * 4) + 5 * round256(2 * V * 4) +
         3 * round256(2 * V * 8);
}

Server::Server(const gn_ens_params &traj, size_t budget, unsigned long long seed, int ntier, const int *tier_blocks,
               const long long *tier_min_volume, int device)
    : device_(device), budget_(budget), seed_(seed), tol_(traj.tol), precision_(traj.precision) {
  if (traj.steps < 1 || traj.integrator < 0 || traj.integrator > 2 || !(traj.tol > 0.0) ||
      (traj.precision != GN_PREC_MIXED && traj.precision != GN_PREC_FP64))
    throw GnError(GN_ERR_ARG, "bad trajectory parameters");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw GnError(GN_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) throw GnError(GN_ERR_ARG, "no such device");
  check(cudaSetDevice(device), "cudaSetDevice");
  cudaDeviceProp prop;
  check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major != 10) throw GnError(GN_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only");
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaMemPoolProps props;
  memset(&props, 0, sizeof props);
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  check(cudaMemPoolCreate(&pool_, &props), "cudaMemPoolCreate");
  uint64_t keep = uint64_t(budget_);
  check(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep), "pool release threshold");
  capacity_ = coop_capacity((const void *)ens_node_kernel, kEnsThreads);
  if (capacity_ < 1) throw GnError(GN_ERR_CUDA, "the batched kernel cannot be resident as a cooperative grid");
  // team tiers: sizes > 1, decreasing, each dividing the previous one (so a
  // block's team in a later tier lies inside its team of the earlier one)
  if (ntier < 0 || ntier > kMaxTiers - 1) throw GnError(GN_ERR_ARG, "0 to 3 team tiers");
  for (int t = 0; t < ntier; t++) {
    const int gs = tier_blocks[t];
    if (gs < 2 || gs > capacity_ || (t > 0 && tier_blocks[t - 1] % gs != 0) ||
        (t > 0 && tier_min_volume[t] > tier_min_volume[t - 1]))
      throw GnError(GN_ERR_ARG, "team tiers: sizes >= 2, each dividing the previous, volumes decreasing");
    tier_gs_.push_back(gs);
    tier_min_.push_back(tier_min_volume[t]);
  }
  // ---- programs: the trajectory (sliced like the ensemble's), a solve, a condensate
  traj_.node_begin = {0};
  ops_ = {{E_REFRESH, 0.0}, {E_PHI, 0.0}, {E_SOLVE, 0.0}, {E_ENERGY0, 0.0}};
  {
    const std::vector<Op> sched = schedule(traj.integrator, traj.eps, traj.steps);
    const int per_node = (traj.integrator == GN_LF2) ? 1 : 2;
    int solves = per_node;
    for (size_t k = 0; k < sched.size(); k++) {
      const Op &o = sched[k];
      std::vector<EnsOp> add;
      if (o.op == OP_F_MED || o.op == OP_F_HIGH) {
        double c = 0.0;
        if (k + 1 < sched.size() && sched[k + 1].op == OP_P) {
          c = sched[k + 1].c;
          k++;
        }
        add = {{E_SOLVE, 0.0}, {E_FORCE, c}};
      } else if (o.op == OP_P) {
        add = {{E_P, o.c}};
      } else if (o.op == OP_Q) {
        add = {{E_Q, o.c}};
      } else {
        add = {{E_SOLVE, 0.0}};
      }
      if (add[0].code == E_SOLVE) {
        if (solves == per_node) {
          traj_.node_begin.push_back(int(ops_.size()));
          solves = 0;
        }
        solves++;
      }
      ops_.insert(ops_.end(), add.begin(), add.end());
    }
    ops_.push_back({E_ENERGY1, 0.0});
    ops_.push_back({E_METROPOLIS, 0.0});
    traj_.node_begin.push_back(int(ops_.size()));
  }
  solve_.node_begin = {int(ops_.size())};
  ops_.push_back({E_RHS, 0.0});
  ops_.push_back({E_SOLVE, 1.0});
  solve_.node_begin.push_back(int(ops_.size()));
  cond_.node_begin = {int(ops_.size())};
  for (int k = 0; k < kMaxNoise / 2; k++) {  // slice k: noise vectors 2k, 2k+1
    ops_.push_back({E_Z2, double(k)});
    ops_.push_back({E_SOLVE, 2.0});
    ops_.push_back({E_TRACE, 0.0});
    cond_.node_begin.push_back(int(ops_.size()));
  }
  for (Program *pg : {&traj_, &solve_, &cond_}) {
    for (size_t k = 0; k + 1 < pg->node_begin.size(); k++) {
      int n = 0;
      for (int o = pg->node_begin[k]; o < pg->node_begin[k + 1]; o++) n += ops_[o].code == E_SOLVE;
      pg->solves.push_back(n);
    }
  }
  check(cudaMalloc(&d_ops_, ops_.size() * sizeof(EnsOp)), "cudaMalloc ops");
  check(cudaMemcpyAsync(d_ops_, ops_.data(), ops_.size() * sizeof(EnsOp), cudaMemcpyHostToDevice, stream_), "copy");
  check(cudaMalloc(&d_states_, kMaxChains * sizeof(EnsState)), "cudaMalloc states");
  check(cudaMemsetAsync(d_states_, 0, kMaxChains * sizeof(EnsState), stream_), "memset states");
  check(cudaMalloc(&d_table_, kMaxChains * sizeof(EnsChain)), "cudaMalloc table");
  check(cudaHostAlloc((void **)&h_table_, kMaxChains * sizeof(EnsChain), cudaHostAllocDefault), "cudaHostAlloc");
  check(cudaHostAlloc((void **)&h_states_, kMaxChains * sizeof(EnsState), cudaHostAllocDefault), "cudaHostAlloc");
  memset(h_states_, 0, kMaxChains * sizeof(EnsState));
  check(cudaMalloc(&d_order_, kMaxChains * sizeof(int)), "cudaMalloc order");
  check(cudaMalloc(&d_queue_, kMaxTiers * sizeof(int)), "cudaMalloc queue");
  check(cudaMalloc(&d_bars_, size_t(kMaxTiers) * capacity_ * sizeof(PhaseBar)), "cudaMalloc bars");
  // two regions: the teams' partial sums, and those of the second flavour of two-team solves
  check(cudaMalloc(&d_partials_, size_t(2) * kMaxTiers * capacity_ * 2 * (kSyncQ + 1) * sizeof(double)),
        "cudaMalloc partials");
  check(cudaMalloc(&d_cg_state_, size_t(capacity_) * kMaxRhs * sizeof(CgState)), "cudaMalloc cg state");
  check(cudaMalloc(&d_err_, sizeof(int)), "cudaMalloc err");
  check(cudaMemsetAsync(d_err_, 0, sizeof(int), stream_), "memset err");
  check(cudaStreamSynchronize(stream_), "server set-up");
  t0_ = std::chrono::steady_clock::now();
}

Server::~Server() {
  cudaSetDevice(device_);
  cudaStreamSynchronize(stream_);
  for (auto &kv : reqs_)
    if (kv.second.work) cudaFreeAsync(kv.second.work, stream_);
  for (Chain &c : chains_) {
    cudaFree(c.sigma[0]);
    cudaFree(c.sigma[1]);
    cudaFree(c.sm);
  }
  cudaStreamSynchronize(stream_);
  cudaFree(d_ops_);
  cudaFree(d_states_);
  cudaFree(d_table_);
  cudaFreeHost(h_table_);
  cudaFreeHost(h_states_);
  cudaFree(d_order_);
  cudaFree(d_queue_);
  cudaFree(d_bars_);
  cudaFree(d_partials_);
  cudaFree(d_cg_state_);
  cudaFree(d_err_);
  if (pool_) cudaMemPoolDestroy(pool_);
  cudaStreamDestroy(stream_);
}

int Server::add_chain(int L, double beta, const double *sigma, unsigned long long stream_id) {
  if (L < 4 || L > 256 || (L & 1)) throw GnError(GN_ERR_ARG, "L must be even and in [4, 256]");
  if (int(chains_.size()) >= kMaxChains) throw GnError(GN_ERR_ARG, "too many chains");
  if (sigma == nullptr) throw GnError(GN_ERR_ARG, "null sigma");
  Chain c;
  c.L = L;
  c.g = make_geom(L);
  c.w = row_width(L, 4);
  c.beta = beta;
  c.stream = stream_id;
  const size_t V = size_t(c.g.V);
  check(cudaMalloc(&c.sigma[0], V * sizeof(double)), "cudaMalloc sigma");
  check(cudaMalloc(&c.sigma[1], V * sizeof(double)), "cudaMalloc sigma");
  check(cudaMalloc(&c.sm, V * sizeof(double)), "cudaMalloc sm");
  check(cudaMemcpyAsync(c.sigma[0], sigma, V * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload sigma");
  sigma_mass_kernel<double><<<unsigned((V + kOpThreads - 1) / kOpThreads), kOpThreads, 0, stream_>>>(
      c.g, c.sigma[0], nullptr, 0.0, nullptr, c.sm);
  check(cudaGetLastError(), "sigma_mass_kernel");
  check(cudaStreamSynchronize(stream_), "add chain");
  chains_.push_back(c);
  return int(chains_.size()) - 1;
}

long long Server::submit(int chain, int type, int nnoise, double t_arrival) {
  if (chain < 0 || chain >= int(chains_.size())) throw GnError(GN_ERR_ARG, "no such chain");
  Req r;
  memset(&r.info, 0, sizeof r.info);
  r.info.id = next_id_++;
  r.info.type = type;
  r.info.chain = chain;
  r.info.t_arrival = t_arrival;
  r.info.noise_vectors = 0;
  if (type == GN_REQ_TRAJECTORY) {
    r.prog = &traj_;
    r.nslices = int(traj_.node_begin.size()) - 1;
  } else if (type == GN_REQ_SOLVE) {
    r.prog = &solve_;
    r.nslices = 1;
  } else if (type == GN_REQ_CONDENSATE) {
    if (nnoise < 2 || nnoise > kMaxNoise || (nnoise & 1)) throw GnError(GN_ERR_ARG, "noise vectors: even, 2..64");
    r.prog = &cond_;
    r.nslices = nnoise / 2;
    r.info.noise_vectors = nnoise;
  } else {
    throw GnError(GN_ERR_ARG, "unknown request type");
  }
  r.bytes = work_bytes(size_t(chains_[chain].g.V));
  if (r.bytes > budget_) throw GnError(GN_ERR_ARG, "the request's work arrays exceed the memory budget");
  r.serial = chains_[chain].nreq++;
  const long long id = r.info.id;
  reqs_[id] = std::move(r);
  queue_.push_back(id);
  return id;
}

// X of a request's work arrays (the layout of chain_entry below).
double *Server::work_X(const Req &r, size_t V) {
  return reinterpret_cast<double *>(static_cast<char *>(r.work) + 3 * round256(V * 8) + 2 * round256(2 * V * 8));
}

EnsChain Server::chain_entry(const Req &r) {
  const Chain &c = chains_[r.info.chain];
  const size_t V = size_t(c.g.V);
  EnsChain e;
  memset(&e, 0, sizeof e);
  e.state = d_states_ + r.info.chain;
  e.op_begin = r.prog->node_begin[r.next];
  e.op_end = r.prog->node_begin[r.next + r.take];
  e.g = c.g;
  e.w = c.w;
  e.beta_s = c.beta;
  e.stream = c.stream;
  e.sigma[0] = c.sigma[0];
  e.sigma[1] = c.sigma[1];
  e.sm = c.sm;
  char *p = static_cast<char *>(r.work);
  auto dv = [&](int planes) {
    double *q = reinterpret_cast<double *>(p);
    p += round256(planes * V * 8);
    return q;
  };
  auto fv = [&](int planes) {
    float *q = reinterpret_cast<float *>(p);
    p += round256(planes * V * 4);
    return q;
  };
  e.P = dv(1);
  e.F = dv(1);
  e.sigma_save = dv(1);
  e.chi = dv(2);
  e.phi = dv(2);
  e.X = dv(2);
  e.Y = dv(2);
  e.t64 = dv(2);
  e.sm32 = fv(1);
  e.rh = fv(2);
  e.ph = fv(2);
  e.uh = fv(2);
  e.ah = fv(2);
  e.xh = fv(2);
  e.r64 = dv(2);
  e.pa64 = dv(2);
  e.pb64 = dv(2);
  e.precision = precision_;
  return e;
}

// Queued requests in arrival order, skipping those whose chain is busy or that
// do not fit the memory left (a later, smaller one may still fit).
void Server::admit() {
  for (auto it = queue_.begin(); it != queue_.end();) {
    Req &r = reqs_[*it];
    Chain &c = chains_[r.info.chain];
    if (c.busy || in_use_ + r.bytes > budget_) {
      ++it;
      continue;
    }
    check(cudaMallocFromPoolAsync(&r.work, r.bytes, pool_, stream_), "cudaMallocFromPoolAsync work");
    in_use_ += r.bytes;
    c.busy = true;
    // the request's serial number on its chain (its Philox counter) and a zero accumulator
    const unsigned long long serial = r.serial;
    const double zero = 0.0;
    EnsState *st = d_states_ + r.info.chain;
    check(cudaMemcpyAsync(&st->serial, &serial, sizeof serial, cudaMemcpyHostToDevice, stream_), "copy serial");
    check(cudaMemcpyAsync(&st->result, &zero, sizeof zero, cudaMemcpyHostToDevice, stream_), "copy result");
    check(cudaStreamSynchronize(stream_), "admit");  // the host values above are stack variables
    r.info.t_admit = clock();
    r.info.status = 1;
    r.iters0 = h_states_[r.info.chain].iters;  // unchanged since the chain's last request retired
    running_.push_back(*it);
    it = queue_.erase(it);
  }
}

int Server::step() {
  TraceRange tr("gn server step");
  admit();
  if (running_.empty()) return 0;
  // Team size of the top tier this step: the whole GPU shared among the
  // running top-tier requests (at least the configured size, a multiple of the
  // next tier's so the teams nest), so a lone big request gets every SM.
  const int ntier_cfg = int(tier_gs_.size());
  int top = ntier_cfg > 0 ? tier_gs_[0] : 1;
  if (ntier_cfg > 0) {
    int n0 = 0;
    for (long long id : running_) n0 += tier_of(chains_[reqs_[id].info.chain].g.V) == 0 ? 1 : 0;
    const int unit = ntier_cfg > 1 ? tier_gs_[1] : 1;
    const int share = (capacity_ / std::max(1, n0)) / unit * unit;
    top = std::max(top, share);
  }
  auto team_size = [&](int tier) { return tier == 0 ? top : (tier < ntier_cfg ? tier_gs_[tier] : 1); };
  // Slices of this step: the launch lasts about as long as its costliest slice
  // (cost ~ V x solves / team size), so every request takes as many further
  // slices as fit in that time -- small requests finish in one step instead of
  // waiting a step per slice behind a big one.
  auto slice_cost = [&](const Req &r, int k) {
    const double V = double(chains_[r.info.chain].g.V);
    return V * double(std::max(1, r.prog->solves[k])) / double(team_size(tier_of(int64_t(V))));
  };
  double span = 0.0;
  for (long long id : running_) span = std::max(span, slice_cost(reqs_[id], reqs_[id].next));
  std::vector<double> cost(running_.size());
  for (size_t i = 0; i < running_.size(); i++) {
    Req &r = reqs_[running_[i]];
    double c = slice_cost(r, r.next);
    r.take = 1;
    while (r.next + r.take < r.nslices && c + slice_cost(r, r.next + r.take) <= span) c += slice_cost(r, r.next + r.take++);
    cost[i] = c;
  }
  // the launch's chain table: tier by tier, each tier costliest first
  std::vector<int> order(running_.size());
  std::iota(order.begin(), order.end(), 0);
  for (size_t i = 0; i < running_.size(); i++) h_table_[i] = chain_entry(reqs_[running_[i]]);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const int ta = tier_of(h_table_[a].g.V), tb = tier_of(h_table_[b].g.V);
    if (ta != tb) return ta < tb;
    return cost[a] > cost[b];
  });
  const int n = int(running_.size());
  check(cudaMemcpyAsync(d_table_, h_table_, n * sizeof(EnsChain), cudaMemcpyHostToDevice, stream_), "copy table");
  check(cudaMemcpyAsync(d_order_, order.data(), n * sizeof(int), cudaMemcpyHostToDevice, stream_), "copy order");
  check(cudaMemsetAsync(d_queue_, 0, kMaxTiers * sizeof(int), stream_), "memset queue");
  check(cudaMemsetAsync(d_bars_, 0, size_t(kMaxTiers) * capacity_ * sizeof(PhaseBar), stream_), "memset bars");
  EnsLaunch a;
  a.chains = d_table_;
  a.nchains = n;
  a.order = d_order_;
  a.ntier = int(tier_gs_.size()) + 1;
  for (int t = 0; t < a.ntier; t++) {
    a.tier_gs[t] = team_size(t);
    int end = 0;
    for (int i : order)
      if (tier_of(h_table_[i].g.V) <= t) end++;
    a.tier_end[t] = end;
  }
  a.ops = d_ops_;
  a.op_begin = -1;
  a.op_end = -1;
  a.queue = d_queue_;
  a.bars = d_bars_;
  a.partials = d_partials_;
  a.partials2 = d_partials_ + size_t(kMaxTiers) * capacity_ * 2 * (kSyncQ + 1);
  a.duo = ens_duo_enabled();
  a.cg_state = d_cg_state_;
  a.err = d_err_;
  a.seed = seed_;
  a.tol = tol_;
  a.delta = 0.01;
  a.n_ru = 100;
  void *args[] = {(void *)&a};
  check(cudaLaunchCooperativeKernel((const void *)ens_node_kernel, dim3(capacity_), dim3(kEnsThreads), args, 0,
                                    stream_),
        "ens_node_kernel launch");
  int h_err = 0;
  check(cudaMemcpyAsync(&h_err, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy err");
  check(cudaMemcpyAsync(h_states_, d_states_, chains_.size() * sizeof(EnsState), cudaMemcpyDeviceToHost, stream_),
        "copy states");
  check(cudaStreamSynchronize(stream_), "server step");
  if (h_err != 0) {
    cudaMemsetAsync(d_err_, 0, sizeof(int), stream_);
    cudaStreamSynchronize(stream_);
    throw GnError(GN_ERR_TIMEOUT, "server step: a team barrier timed out");
  }
  // retire the finished requests
  int done = 0;
  const double now = clock();
  std::vector<long long> still;
  for (long long id : running_) {
    Req &r = reqs_[id];
    r.next += r.take;
    if (r.next < r.nslices) {
      still.push_back(id);
      continue;
    }
    const EnsState &s = h_states_[r.info.chain];
    Chain &c = chains_[r.info.chain];
    r.info.failed = s.failed;
    if (r.info.type == GN_REQ_TRAJECTORY) {
      r.info.dH = s.last_dH;
      r.info.accepted = s.last_acc;
    } else if (r.info.type == GN_REQ_CONDENSATE) {
      r.info.value = s.result / double(r.info.noise_vectors);
    } else {
      const size_t V = size_t(c.g.V);
      r.x.resize(V);
      check(cudaMemcpyAsync(r.x.data(), work_X(r, V), V * sizeof(double), cudaMemcpyDeviceToHost, stream_),
            "copy x");
      check(cudaStreamSynchronize(stream_), "copy x");
    }
    r.info.cg_iterations = s.iters - r.iters0;
    check(cudaFreeAsync(r.work, stream_), "cudaFreeAsync work");
    r.work = nullptr;
    in_use_ -= r.bytes;
    c.busy = false;
    r.info.t_done = now;
    r.info.status = 2;
    done++;
  }
  running_.swap(still);
  return done;
}

void Server::request(long long id, gn_request_info *out) {
  auto it = reqs_.find(id);
  if (it == reqs_.end()) throw GnError(GN_ERR_ARG, "no such request");
  *out = it->second.info;
}

void Server::solution(long long id, double *x) {
  auto it = reqs_.find(id);
  if (it == reqs_.end()) throw GnError(GN_ERR_ARG, "no such request");
  const Req &r = it->second;
  if (r.info.type != GN_REQ_SOLVE || r.info.status != 2) throw GnError(GN_ERR_ARG, "not a finished solve");
  memcpy(x, r.x.data(), r.x.size() * sizeof(double));
}

void Server::chain_sigma(int chain, double *sigma) {
  if (chain < 0 || chain >= int(chains_.size())) throw GnError(GN_ERR_ARG, "no such chain");
  const Chain &c = chains_[chain];
  int cur = 0;
  check(cudaMemcpyAsync(&cur, &d_states_[chain].cur, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "sync");
  check(cudaMemcpyAsync(sigma, c.sigma[cur], size_t(c.g.V) * sizeof(double), cudaMemcpyDeviceToHost, stream_),
        "copy sigma");
  check(cudaStreamSynchronize(stream_), "chain sigma");
}

void Server::load(int *running, int *queued, long long *bytes) {
  if (running) *running = int(running_.size());
  if (queued) *queued = int(queue_.size());
  if (bytes) *bytes = (long long)in_use_;
}

}  // namespace gn

struct gn_server {
  std::unique_ptr<gn::Server> s;
};

namespace {

template <typename F>
long long srv_guarded(gn_server *s, F &&f) {
  if (s == nullptr || !s->s) return gn::set_last_error(GN_ERR_ARG, "null server");
  try {
    cudaSetDevice(s->s->device());
    return f(*s->s);
  } catch (const gn::GnError &x) {
    return gn::set_last_error(x.status, x.what());
  } catch (const std::exception &x) {
    return gn::set_last_error(GN_ERR_CUDA, x.what());
  }
}

}  // namespace

extern "C" {

int gn_server_create(gn_server **out, const gn_ens_params *traj, double mem_budget_bytes, unsigned long long seed,
                     int ntiers, const int *tier_blocks, const long long *tier_min_volume, int device) {
  if (out == nullptr || traj == nullptr) return gn::set_last_error(GN_ERR_ARG, "null argument");
  if (ntiers > 0 && (tier_blocks == nullptr || tier_min_volume == nullptr))
    return gn::set_last_error(GN_ERR_ARG, "null tier arrays");
  *out = nullptr;
  if (!(mem_budget_bytes > 0)) return gn::set_last_error(GN_ERR_ARG, "memory budget must be positive");
  try {
    auto s = std::make_unique<gn_server>();
    s->s = std::make_unique<gn::Server>(*traj, size_t(mem_budget_bytes), seed, ntiers, tier_blocks, tier_min_volume,
                                        device);
    *out = s.release();
    return GN_OK;
  } catch (const gn::GnError &x) {
    return gn::set_last_error(x.status, x.what());
  } catch (const std::exception &x) {
    return gn::set_last_error(GN_ERR_CUDA, x.what());
  }
}

void gn_server_destroy(gn_server *s) { delete s; }

int gn_server_add_chain(gn_server *s, int L, double beta_s, const double *sigma, unsigned long long stream_id) {
  return int(srv_guarded(s, [&](gn::Server &S) { return (long long)S.add_chain(L, beta_s, sigma, stream_id); }));
}

double gn_server_clock(gn_server *s) { return (s && s->s) ? s->s->clock() : 0.0; }

long long gn_server_submit(gn_server *s, int chain, int type, int noise_vectors, double t_arrival) {
  return srv_guarded(s, [&](gn::Server &S) { return S.submit(chain, type, noise_vectors, t_arrival); });
}

int gn_server_step(gn_server *s, int *completed) {
  return int(srv_guarded(s, [&](gn::Server &S) {
    const int d = S.step();
    if (completed) *completed = d;
    return (long long)GN_OK;
  }));
}

int gn_server_request(gn_server *s, long long id, gn_request_info *out) {
  if (out == nullptr) return gn::set_last_error(GN_ERR_ARG, "null output");
  return int(srv_guarded(s, [&](gn::Server &S) {
    S.request(id, out);
    return (long long)GN_OK;
  }));
}

int gn_server_solution(gn_server *s, long long id, double *x) {
  if (x == nullptr) return gn::set_last_error(GN_ERR_ARG, "null output");
  return int(srv_guarded(s, [&](gn::Server &S) {
    S.solution(id, x);
    return (long long)GN_OK;
  }));
}

int gn_server_chain_sigma(gn_server *s, int chain, double *sigma) {
  if (sigma == nullptr) return gn::set_last_error(GN_ERR_ARG, "null output");
  return int(srv_guarded(s, [&](gn::Server &S) {
    S.chain_sigma(chain, sigma);
    return (long long)GN_OK;
  }));
}

int gn_server_load(gn_server *s, int *running, int *queued, long long *bytes_in_use) {
  return int(srv_guarded(s, [&](gn::Server &S) {
    S.load(running, queued, bytes_in_use);
    return (long long)GN_OK;
  }));
}

}  // extern "C"
