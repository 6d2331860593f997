// Batched ensembles of independent channels on one GPU.  No counterpart in
// the reference: its main loop (src/main.cc:114-154) runs one channel.  Each
// member is an ordinary context (its own parameters, fields, solver tables
// and tuned FFT tiles); one ensemble step is ONE graph launch whose branches
// are the members' fused steps, so small members that cannot fill 148 SMs
// alone run side by side.  Between two steps that need the host (checks, a
// new CFL-controlled dt) the members need not meet: one launch of a second
// graph runs K steps, each branch a member's K steps in a row, so members
// that finish early leave the GPU to the others instead of waiting for the
// largest at every step.  Members are scheduled in groups (the members of a
// group run concurrently, groups one after another), and every member's
// persistent kernels get an SM budget.  The batched schedule instead walks
// the step stage by stage: each stage of the mixed-form members is ONE
// launch over a work list of (member, tile) items -- its blocks fill the
// device with tiles of all the members, so small members no longer run at
// the latency of their own short kernels -- and the transforms take one
// launch per line length (their plans are compiled per length), run
// concurrently.  An autotuner times the candidate schedules on the members'
// own fields and keeps the fastest.  Checks, CFL-controlled dt and the
// device error word stay per member, as in plc_step.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "plc_internal.h"

struct plc_ensemble {
  int device = 0;
  std::vector<plc_ctx *> members;
  cudaStream_t stream = nullptr;  // graph launches
  cudaEvent_t fork = nullptr, done = nullptr, t0 = nullptr, t1 = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph = nullptr;
  cudaGraphExec_t graph_k = nullptr;   // K steps per branch
  cudaGraphExec_t graph_kc = nullptr;  // K steps ending on a check step, with the checks
  int k_steps = 0;
  std::vector<unsigned> epochs;     // member graph epochs the graph was captured at
  std::vector<unsigned> epochs_k;   // ... and the K-step graphs
  std::vector<unsigned> epochs_kc;
  std::vector<int> group;        // group of each member
  int ngroups = 1;
  int scheme = PLC_ENS_CONCURRENT;
  std::vector<double> cost;  // measured ms per step of each member alone (0 = not measured)
  // PLC_ENS_BATCHED: streams (and their join events) of the concurrent
  // launches of a batched transform stage, one per line length
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> aux_join;
  // PLC_ENS_BATCHED with two chains: the second chain's stream, its fork from
  // the ensemble stream and its join, and the fork events of both chains'
  // batched transform stages
  cudaStream_t chain_stream = nullptr;
  cudaEvent_t chain_join = nullptr;
  cudaEvent_t stage_fork[2] = {nullptr, nullptr};
  int chains = 1;        // batched chains of mixed-form members, run concurrently (1 or 2)
  plc::BatchPlan bplan;  // families, tiles and z chunk of the batched launches
  std::string err;
};

namespace {

std::string g_ens_err;

int ens_error(plc_ensemble *e, int code, const std::string &msg) {
  if (e) e->err = msg;
  g_ens_err = msg;
  return code;
}

int ens_cuda(plc_ensemble *e, cudaError_t r, const char *what) {
  return ens_error(e, PLC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(r));
}

#define ENS_CUDA(e, call)                                   \
  do {                                                      \
    cudaError_t _r = (call);                                \
    if (_r != cudaSuccess) return ens_cuda(e, _r, #call);   \
  } while (0)

// a member's failure, reported with the member's index and message
int member_error(plc_ensemble *e, int m, int rc) {
  return ens_error(e, rc, "member " + std::to_string(m) + ": " + plc_last_error(e->members[m]));
}

void drop(plc_ensemble *e) {
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  if (e->graph_k) {
    cudaGraphExecDestroy(e->graph_k);
    e->graph_k = nullptr;
  }
  if (e->graph_kc) {
    cudaGraphExecDestroy(e->graph_kc);
    e->graph_kc = nullptr;
  }
}

constexpr int kAuxStreams = 8;

// One batched transform stage of a chain: its launches (one per line
// length) on the chain's auxiliary streams aux[a0 .. a0+na), forked from and
// joined to the chain's stream st.
template <class F>
cudaError_t batched_stage(plc_ensemble *e, cudaStream_t st, cudaEvent_t fork, int a0, int na,
                          int groups, F &&launch) {
  if (groups <= 1 || na <= 1) return launch(&st, 1);
  na = std::min(groups, na);
  cudaError_t r = cudaEventRecord(fork, st);
  for (int a = a0; a < a0 + na && r == cudaSuccess; ++a) r = cudaStreamWaitEvent(e->aux[a], fork, 0);
  if (r == cudaSuccess) r = launch(e->aux.data() + a0, na);
  for (int a = a0; a < a0 + na && r == cudaSuccess; ++a) {
    if ((r = cudaEventRecord(e->aux_join[a], e->aux[a])) == cudaSuccess)
      r = cudaStreamWaitEvent(st, e->aux_join[a], 0);
  }
  return r;
}

// `steps` steps of the mixed-form channels cs[0..n) stage by stage on stream
// st, each stage one launch over all of them (the transforms: one per line
// length, concurrently on aux[a0 .. a0+na)).
int enqueue_chain(plc_ensemble *e, plc_ctx *const *cs, int n, int steps, cudaStream_t st,
                  cudaEvent_t fork, int a0, int na) {
  const int gx = plc::fft_batch_groups(cs, n, false), gy = plc::fft_batch_groups(cs, n, true);
  const int kc = e->bplan.rk_kchunk, mb = e->bplan.rk_minb;
  const plc::BatchPlan *bp = &e->bplan;
  const bool pdl = bp->pdl;
  for (int q = 0; q < steps; ++q) {
    ENS_CUDA(e, plc::launch_rk_batch(cs, n, 1, kc, mb, st, pdl));  // RK1 + bound(u1)
    ENS_CUDA(e, plc::launch_rk_batch(cs, n, 2, kc, mb, st, pdl));  // RK2 + bound(u) + forcing
    ENS_CUDA(e, batched_stage(e, st, fork, a0, na, gx, [&](const cudaStream_t *ss, int ns) {
               return plc::launch_fft_x_fwd_batch(cs, n, bp, ss, ns);  // calcRHS + x-FFT
             }));
    ENS_CUDA(e, batched_stage(e, st, fork, a0, na, gy, [&](const cudaStream_t *ss, int ns) {
               return plc::launch_fft_y_batch(cs, n, false, bp, ss, ns);  // y-FFT
             }));
    ENS_CUDA(e, plc::launch_trid_batch(cs, n, bp->trid_tile, st, pdl));  // z solve
    ENS_CUDA(e, batched_stage(e, st, fork, a0, na, gy, [&](const cudaStream_t *ss, int ns) {
               return plc::launch_fft_y_batch(cs, n, true, bp, ss, ns);  // y-iFFT
             }));
    ENS_CUDA(e, batched_stage(e, st, fork, a0, na, gx, [&](const cudaStream_t *ss, int ns) {
               return plc::launch_fft_x_bwd_batch(cs, n, bp, ss, ns);  // x-iFFT + bound(p)
             }));
    ENS_CUDA(e, plc::launch_correct_batch(cs, n, st, pdl));  // correct + force + bound(u)
  }
  return PLC_OK;
}

// The PLC_ENS_BATCHED form of `steps` ensemble steps (inside a capture on the
// ensemble stream): the FP64 members' fused steps as branches; the
// mixed-form members in e->chains chains (cost-balanced, longest first),
// each chain's steps stage by stage, the chains concurrently.
int enqueue_batched(plc_ensemble *e, int steps, bool checks) {
  std::vector<int> mixed, fp64;
  for (size_t m = 0; m < e->members.size(); ++m) (e->members[m]->mixed ? mixed : fp64).push_back((int)m);
  ENS_CUDA(e, cudaEventRecord(e->fork, e->stream));
  for (int m : fp64) {
    plc_ctx *c = e->members[m];
    ENS_CUDA(e, cudaStreamWaitEvent(c->stream, e->fork, 0));
    for (int q = 0; q < steps; ++q)
      if (int rc = plc::capture_step(c, c->stream)) return member_error(e, m, rc);
    if (checks)
      if (int rc = plc::enqueue_check_tail(c, c->stream)) return member_error(e, m, rc);
    ENS_CUDA(e, cudaEventRecord(e->join[m], c->stream));
  }
  const int nch = (int)mixed.size() >= 2 ? e->chains : 1;
  std::vector<plc_ctx *> chain[2];
  {
    std::vector<int> order = mixed;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->cost[a] > e->cost[b]; });
    double load[2] = {0.0, 0.0};
    for (int m : order) {
      const int k = (nch == 2 && load[1] < load[0]) ? 1 : 0;
      chain[k].push_back(e->members[m]);
      load[k] += e->cost[m];
    }
  }
  if (nch == 2) {
    ENS_CUDA(e, cudaStreamWaitEvent(e->chain_stream, e->fork, 0));
    if (int rc = enqueue_chain(e, chain[1].data(), (int)chain[1].size(), steps, e->chain_stream,
                               e->stage_fork[1], kAuxStreams / 2, kAuxStreams / 2))
      return rc;
    ENS_CUDA(e, cudaEventRecord(e->chain_join, e->chain_stream));
  }
  if (!chain[0].empty())
    if (int rc = enqueue_chain(e, chain[0].data(), (int)chain[0].size(), steps, e->stream,
                               e->stage_fork[0], 0, nch == 2 ? kAuxStreams / 2 : kAuxStreams))
      return rc;
  if (nch == 2) ENS_CUDA(e, cudaStreamWaitEvent(e->stream, e->chain_join, 0));
  if (checks && !mixed.empty()) {
    // the mixed-form members' checks and new dt in one launch
    std::vector<plc_ctx *> ms;
    for (int m : mixed) ms.push_back(e->members[m]);
    ENS_CUDA(e, plc::launch_check_batch(ms.data(), (int)ms.size(), e->stream, e->bplan.pdl));
  }
  for (int m : fp64) ENS_CUDA(e, cudaStreamWaitEvent(e->stream, e->join[m], 0));
  return PLC_OK;
}

// Captures `steps` ensemble steps into *out: per group, a fork from the
// ensemble stream to the members' streams, each member's fused steps in a
// row (with `checks`, then its full check and CFL-controlled dt), a join
// back (PLC_ENS_BATCHED: enqueue_batched).
int capture(plc_ensemble *e, int steps, cudaGraphExec_t *out, std::vector<unsigned> &epochs,
            bool checks = false) {
  const int n = (int)e->members.size();
  bool stale = *out == nullptr;
  for (int m = 0; m < n && !stale; ++m) stale = epochs[m] != e->members[m]->graph_epoch;
  if (!stale) return PLC_OK;
  if (*out) {
    cudaGraphExecDestroy(*out);
    *out = nullptr;
  }
  for (int m = 0; m < n; ++m)
    if (!e->members[m]->poisson_ready)
      return ens_error(e, PLC_ERR_STATE, "member " + std::to_string(m) + ": Poisson solver not initialised");
  cudaGraph_t g = nullptr;
  ENS_CUDA(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  int rc = PLC_OK;
  cudaError_t r = cudaSuccess;
  if (e->scheme == PLC_ENS_BATCHED) rc = enqueue_batched(e, steps, checks);
  for (int grp = 0; grp < e->ngroups && rc == PLC_OK && r == cudaSuccess &&
                    e->scheme != PLC_ENS_BATCHED;
       ++grp) {
    if ((r = cudaEventRecord(e->fork, e->stream)) != cudaSuccess) break;
    for (int m = 0; m < n && rc == PLC_OK && r == cudaSuccess; ++m) {
      if (e->group[m] != grp) continue;
      plc_ctx *c = e->members[m];
      if ((r = cudaStreamWaitEvent(c->stream, e->fork, 0)) != cudaSuccess) break;
      for (int q = 0; q < steps && rc == PLC_OK; ++q)
        if ((rc = plc::capture_step(c, c->stream)) != PLC_OK) rc = member_error(e, m, rc);
      if (rc == PLC_OK && checks && (rc = plc::enqueue_check_tail(c, c->stream)) != PLC_OK)
        rc = member_error(e, m, rc);
      if (rc != PLC_OK) break;
      r = cudaEventRecord(e->join[m], c->stream);
    }
    for (int m = 0; m < n && rc == PLC_OK && r == cudaSuccess; ++m)
      if (e->group[m] == grp) r = cudaStreamWaitEvent(e->stream, e->join[m], 0);
  }
  const cudaError_t re = cudaStreamEndCapture(e->stream, &g);
  if (rc != PLC_OK || r != cudaSuccess || re != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (rc != PLC_OK) return rc;
    return ens_cuda(e, r != cudaSuccess ? r : re, "ensemble step capture");
  }
  r = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (r != cudaSuccess) return ens_cuda(e, r, "cudaGraphInstantiate");
  // the graph's first launch would otherwise carry its upload to the device
  ENS_CUDA(e, cudaGraphUpload(*out, e->stream));
  for (int m = 0; m < n; ++m) epochs[m] = e->members[m]->graph_epoch;
  return PLC_OK;
}

int build(plc_ensemble *e) { return capture(e, 1, &e->graph, e->epochs); }

// K of the multi-step graph: when the members share one check period, that
// period if it is at most kMaxBlockSteps steps, else its largest divisor
// between 8 and kMaxBlockSteps (25 for the reference's nt_check = 100), so
// that every check step ends a block; otherwise 8.  The cap bounds the
// captured graph: its nodes grow with K.
constexpr int kMaxBlockSteps = 32;
int k_of(const plc_ensemble *e) {
  int k = e->members[0]->prm.nt_check;
  for (const plc_ctx *c : e->members)
    if (c->prm.nt_check != k) k = 0;
  if (k > 1 && k <= kMaxBlockSteps) return k;
  if (k > kMaxBlockSteps)
    for (int d = kMaxBlockSteps; d >= 8; --d)
      if (k % d == 0) return d;
  return 8;
}

// Steps, at most `limit`, until (and including) the next step that needs the
// host for any member: 1 when the next step itself does.
int steps_to_host(const plc_ensemble *e, int limit) {
  int best = limit;
  for (const plc_ctx *c : e->members) {
    const plc_params &P = c->prm;
    for (int j = 1; j < best; ++j) {
      const long long n = c->nstep + j;
      const bool host = (P.cfl_target > 0.0 && n < P.nt_check && (n & (n - 1)) == 0) ||
                        (P.nt_check > 0 && n % P.nt_check == 0);
      if (host) {
        best = j;
        break;
      }
    }
  }
  return best;
}

// orders the ensemble stream after all work queued on the members' streams
int ens_after_members(plc_ensemble *e) {
  for (size_t m = 0; m < e->members.size(); ++m) {
    ENS_CUDA(e, cudaEventRecord(e->join[m], e->members[m]->stream));
    ENS_CUDA(e, cudaStreamWaitEvent(e->stream, e->join[m], 0));
  }
  return PLC_OK;
}

// orders the members' streams after the work queued on the ensemble stream
int members_after_ens(plc_ensemble *e) {
  ENS_CUDA(e, cudaEventRecord(e->done, e->stream));
  for (plc_ctx *c : e->members) ENS_CUDA(e, cudaStreamWaitEvent(c->stream, e->done, 0));
  return PLC_OK;
}

int ens_steps(plc_ensemble *e, int nsteps, double *ms) {
  if (nsteps < 0) return ens_error(e, PLC_ERR_ARG, "nsteps < 0");
  const int n = (int)e->members.size();
  const int K = k_of(e);
  if (K != e->k_steps) drop(e);
  e->k_steps = K;
  if (int rc = build(e)) return rc;
  if (int rc = capture(e, K, &e->graph_k, e->epochs_k)) return rc;
  // the block that ends on every member's check step carries the checks
  // (and the CFL-controlled dt) in the graph itself
  bool kc_possible = true;
  for (const plc_ctx *c : e->members)
    kc_possible = kc_possible && c->prm.nt_check > 0 && c->prm.nt_check % K == 0;
  if (kc_possible)
    if (int rc = capture(e, K, &e->graph_kc, e->epochs_kc, true)) return rc;
  for (int m = 0; m < n; ++m)
    if (int rc = plc::pre_steps(e->members[m])) return member_error(e, m, rc);
  if (int rc = ens_after_members(e)) return rc;
  if (ms) ENS_CUDA(e, cudaEventRecord(e->t0, e->stream));
  for (int s = 0; s < nsteps;) {
    // K steps in one launch when none before the block's last needs the host
    const bool block = nsteps - s >= K && steps_to_host(e, K) == K;
    const int q = block ? K : 1;
    bool host = false;
    for (plc_ctx *c : e->members) {
      c->nstep += q - 1;  // the last step of the launch decides
      host = host || plc::step_needs_host(c);
      c->nstep -= q - 1;
    }
    bool dev_checks = block && kc_possible;
    for (const plc_ctx *c : e->members) dev_checks = dev_checks && plc::device_check_due(c, K);
    if (dev_checks) {
      // one launch and one wait for the K steps and every member's check
      ENS_CUDA(e, cudaGraphLaunch(e->graph_kc, e->stream));
      ENS_CUDA(e, cudaStreamSynchronize(e->stream));
      for (int m = 0; m < n; ++m)
        if (int rc = plc::post_steps_device_check(e->members[m], K)) return member_error(e, m, rc);
      s += q;
      continue;
    }
    ENS_CUDA(e, cudaGraphLaunch(block ? e->graph_k : e->graph, e->stream));
    if (host)
      if (int rc = members_after_ens(e)) return rc;
    for (int r = 0; r < q; ++r) {
      // the members' checks queued first, then one wait for all of them
      for (int m = 0; m < n; ++m)
        if (int rc = plc::post_step_begin(e->members[m])) return member_error(e, m, rc);
      for (int m = 0; m < n; ++m)
        if (int rc = plc::post_step_end(e->members[m])) return member_error(e, m, rc);
    }
    // a member's host work ends with a new dt copied on its stream: the next
    // launch is queued after it
    if (host)
      if (int rc = ens_after_members(e)) return rc;
    s += q;
  }
  if (ms) {
    ENS_CUDA(e, cudaEventRecord(e->t1, e->stream));
    ENS_CUDA(e, cudaEventSynchronize(e->t1));
    float t = 0.f;
    ENS_CUDA(e, cudaEventElapsedTime(&t, e->t0, e->t1));
    *ms = t;
  }
  if (int rc = members_after_ens(e)) return rc;
  // the device error word of each member (bounded waits that gave up)
  for (int m = 0; m < n; ++m)
    if (int rc = plc_sync(e->members[m])) return member_error(e, m, rc);
  return PLC_OK;
}

// Device copies of the members' u, v, w, p (the state an autotuning run
// advances), restored afterwards.
struct Snapshot {
  std::vector<void *> buf;
  ~Snapshot() {
    for (void *p : buf) cudaFree(p);
  }
};

const int kStateFields[4] = {PLC_U, PLC_V, PLC_W, PLC_P};

void *field_of(plc_ctx *c, int f) {
  return c->mixed ? static_cast<void *>(c->f_field[f]) : static_cast<void *>(c->d_field[f]);
}
size_t field_bytes(const plc_ctx *c) { return c->nfield * (c->mixed ? sizeof(float) : sizeof(double)); }

int snapshot(plc_ensemble *e, Snapshot &s, bool save) {
  size_t q = 0;
  for (plc_ctx *c : e->members)
    for (int f : kStateFields) {
      if (save) {
        void *p = nullptr;
        ENS_CUDA(e, cudaMalloc(&p, field_bytes(c)));
        s.buf.push_back(p);
        ENS_CUDA(e, cudaMemcpyAsync(p, field_of(c, f), field_bytes(c), cudaMemcpyDeviceToDevice, c->stream));
      } else {
        ENS_CUDA(e, cudaMemcpyAsync(field_of(c, f), s.buf[q++], field_bytes(c), cudaMemcpyDeviceToDevice,
                                    c->stream));
      }
    }
  for (plc_ctx *c : e->members) ENS_CUDA(e, cudaStreamSynchronize(c->stream));
  return PLC_OK;
}

// launches only (no checks, no step counting): the timing loop of the autotuner
int time_launches(plc_ensemble *e, int steps, float *ms) {
  if (int rc = build(e)) return rc;
  if (int rc = ens_after_members(e)) return rc;
  ENS_CUDA(e, cudaGraphLaunch(e->graph, e->stream));  // warm-up
  ENS_CUDA(e, cudaEventRecord(e->t0, e->stream));
  for (int s = 0; s < steps; ++s) ENS_CUDA(e, cudaGraphLaunch(e->graph, e->stream));
  ENS_CUDA(e, cudaEventRecord(e->t1, e->stream));
  ENS_CUDA(e, cudaEventSynchronize(e->t1));
  ENS_CUDA(e, cudaEventElapsedTime(ms, e->t0, e->t1));
  return members_after_ens(e);
}

// a member alone: its own captured step replayed on its stream (launches
// only: no checks, no step counting)
int time_member(plc_ensemble *e, int m, int steps, float *ms) {
  plc_ctx *c = e->members[m];
  cudaGraphExec_t g = nullptr;
  if (int rc = plc::step_graph(c, &g)) return member_error(e, m, rc);
  ENS_CUDA(e, cudaGraphLaunch(g, c->stream));  // warm-up
  ENS_CUDA(e, cudaEventRecord(e->t0, c->stream));
  for (int s = 0; s < steps; ++s) ENS_CUDA(e, cudaGraphLaunch(g, c->stream));
  ENS_CUDA(e, cudaEventRecord(e->t1, c->stream));
  ENS_CUDA(e, cudaEventSynchronize(e->t1));
  float t = 0.f;
  ENS_CUDA(e, cudaEventElapsedTime(&t, e->t0, e->t1));
  *ms = t / steps;
  return PLC_OK;
}

// Applies a schedule: SM budgets per member and the grouping.
int apply_scheme(plc_ensemble *e, int scheme) {
  const int n = (int)e->members.size();
  const int sms = e->members[0]->device_sms;
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->cost[a] > e->cost[b]; });
  e->group.assign(n, 0);
  e->ngroups = 1;
  std::vector<int> budget(n, sms);
  const double total = std::accumulate(e->cost.begin(), e->cost.end(), 0.0);
  switch (scheme) {
    case PLC_ENS_CONCURRENT:  // all members at once, full budgets
      break;
    case PLC_ENS_PROPORTIONAL:  // all at once, SMs shared in proportion to cost
      for (int m = 0; m < n; ++m)
        budget[m] = std::max(1, (int)std::lround(sms * (total > 0 ? e->cost[m] / total : 1.0 / n)));
      break;
    case PLC_ENS_TWO_GROUPS: {  // two cost-balanced groups (LPT), proportional within each
      double load[2] = {0.0, 0.0};
      for (int m : order) {
        const int g = load[0] <= load[1] ? 0 : 1;
        e->group[m] = g;
        load[g] += e->cost[m];
      }
      e->ngroups = 2;
      for (int m = 0; m < n; ++m) {
        const double l = load[e->group[m]];
        budget[m] = std::max(1, (int)std::lround(sms * (l > 0 ? e->cost[m] / l : 1.0)));
      }
      break;
    }
    case PLC_ENS_SEQUENTIAL:  // one member after another, full budgets
      for (int q = 0; q < n; ++q) e->group[order[q]] = q;
      e->ngroups = n;
      break;
    case PLC_ENS_BATCHED: {  // stage by stage over the mixed-form members, full budgets
      bool any = false;
      for (const plc_ctx *c : e->members) any = any || c->mixed;
      if (!any) return ens_error(e, PLC_ERR_ARG, "the batched schedule needs mixed-form members");
      break;
    }
    default:
      return ens_error(e, PLC_ERR_ARG, "unknown ensemble schedule");
  }
  for (int m = 0; m < n; ++m)
    if (int rc = plc_set_sm_budget(e->members[m], budget[m])) return member_error(e, m, rc);
  e->scheme = scheme;
  drop(e);
  return PLC_OK;
}

}  // namespace

using namespace plc;

extern "C" {

const char *plc_ensemble_last_error(const plc_ensemble *e) { return e ? e->err.c_str() : g_ens_err.c_str(); }

int plc_ensemble_create(int n, const plc_params *prms, const double *const *dzf_globals, int device,
                        plc_ensemble **out) {
  if (!out || !prms || n < 1) return ens_error(nullptr, PLC_ERR_ARG, "bad argument");
  *out = nullptr;
  plc_ensemble *e = new plc_ensemble;
  e->device = device;
  auto fail = [&](int rc) {
    const std::string msg = e->err;
    plc_ensemble_destroy(e);
    return ens_error(nullptr, rc, msg);
  };
  for (int m = 0; m < n; ++m) {
    plc_ctx *c = nullptr;
    const int rc = plc_create(&prms[m], dzf_globals ? dzf_globals[m] : nullptr, device, &c);
    if (rc != PLC_OK) {
      e->err = "member " + std::to_string(m) + ": " + plc_last_error(nullptr);
      return fail(rc);
    }
    e->members.push_back(c);
  }
  cudaError_t r;
  if ((r = cudaSetDevice(device)) != cudaSuccess ||
      (r = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (r = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming)) != cudaSuccess ||
      (r = cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming)) != cudaSuccess ||
      (r = cudaEventCreate(&e->t0)) != cudaSuccess || (r = cudaEventCreate(&e->t1)) != cudaSuccess) {
    ens_cuda(e, r, "ensemble stream/events");
    return fail(PLC_ERR_CUDA);
  }
  e->join.assign(n, nullptr);
  for (auto &ev : e->join)
    if ((r = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) {
      ens_cuda(e, r, "ensemble events");
      return fail(PLC_ERR_CUDA);
    }
  if ((r = cudaStreamCreateWithFlags(&e->chain_stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (r = cudaEventCreateWithFlags(&e->chain_join, cudaEventDisableTiming)) != cudaSuccess ||
      (r = cudaEventCreateWithFlags(&e->stage_fork[0], cudaEventDisableTiming)) != cudaSuccess ||
      (r = cudaEventCreateWithFlags(&e->stage_fork[1], cudaEventDisableTiming)) != cudaSuccess) {
    ens_cuda(e, r, "ensemble chain stream/events");
    return fail(PLC_ERR_CUDA);
  }
  e->aux.assign(kAuxStreams, nullptr);
  e->aux_join.assign(kAuxStreams, nullptr);
  for (int a = 0; a < kAuxStreams; ++a)
    if ((r = cudaStreamCreateWithFlags(&e->aux[a], cudaStreamNonBlocking)) != cudaSuccess ||
        (r = cudaEventCreateWithFlags(&e->aux_join[a], cudaEventDisableTiming)) != cudaSuccess) {
      ens_cuda(e, r, "ensemble auxiliary streams");
      return fail(PLC_ERR_CUDA);
    }
  e->epochs.assign(n, ~0u);
  e->epochs_k.assign(n, ~0u);
  e->epochs_kc.assign(n, ~0u);
  e->group.assign(n, 0);
  // cost model before measurement: grid points (FP32 fields move half the bytes)
  e->cost.resize(n);
  for (int m = 0; m < n; ++m) {
    const plc_ctx *c = e->members[m];
    e->cost[m] = double(c->nx) * c->ny * c->nz * (c->mixed ? 0.5 : 1.0);
  }
  *out = e;
  return PLC_OK;
}

int plc_ensemble_destroy(plc_ensemble *e) {
  if (!e) return PLC_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop(e);
  for (plc_ctx *c : e->members) plc_destroy(c);
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {e->fork, e->done, e->t0, e->t1})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : e->aux_join)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {e->chain_join, e->stage_fork[0], e->stage_fork[1]})
    if (ev) cudaEventDestroy(ev);
  if (e->chain_stream) cudaStreamDestroy(e->chain_stream);
  for (cudaStream_t st : e->aux)
    if (st) cudaStreamDestroy(st);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return PLC_OK;
}

int plc_ensemble_size(const plc_ensemble *e, int *n) {
  if (!e || !n) return ens_error(nullptr, PLC_ERR_ARG, "null argument");
  *n = (int)e->members.size();
  return PLC_OK;
}

int plc_ensemble_member(plc_ensemble *e, int i, plc_ctx **ctx) {
  if (!e || !ctx) return ens_error(nullptr, PLC_ERR_ARG, "null argument");
  if (i < 0 || i >= (int)e->members.size()) return ens_error(e, PLC_ERR_ARG, "member index out of range");
  *ctx = e->members[i];
  return PLC_OK;
}

int plc_ensemble_init_flow(plc_ensemble *e) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  for (size_t m = 0; m < e->members.size(); ++m)
    if (int rc = plc_init_flow(e->members[m])) return member_error(e, (int)m, rc);
  return PLC_OK;
}

int plc_ensemble_step(plc_ensemble *e, int nsteps) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  return ens_steps(e, nsteps, nullptr);
}

int plc_ensemble_step_timed(plc_ensemble *e, int nsteps, double *ms) {
  if (!e || !ms) return ens_error(e, PLC_ERR_ARG, "null argument");
  return ens_steps(e, nsteps, ms);
}

int plc_ensemble_set_schedule(plc_ensemble *e, int scheme) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  return apply_scheme(e, scheme);
}

int plc_ensemble_schedule(const plc_ensemble *e, int *scheme, int *groups, int *sm_budgets) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  if (scheme) *scheme = e->scheme;
  if (groups)
    for (size_t m = 0; m < e->members.size(); ++m) groups[m] = e->group[m];
  if (sm_budgets)
    for (size_t m = 0; m < e->members.size(); ++m) sm_budgets[m] = e->members[m]->num_sms;
  return PLC_OK;
}

int plc_ensemble_autotune(plc_ensemble *e, int steps, float *ms_per_scheme) {
  if (!e || steps < 1) return ens_error(e, PLC_ERR_ARG, "bad argument");
  const int n = (int)e->members.size();
  Snapshot snap;
  if (int rc = snapshot(e, snap, true)) return rc;
  int rc = PLC_OK;
  bool any_mixed = false;
  for (const plc_ctx *c : e->members) any_mixed = any_mixed || c->mixed;
  // 1. cost model: each member's step time alone, full budget
  for (int m = 0; m < n && rc == PLC_OK; ++m) {
    if ((rc = plc_set_sm_budget(e->members[m], e->members[m]->device_sms)) != PLC_OK) {
      rc = member_error(e, m, rc);
      break;
    }
    float t = 0.f;
    if ((rc = time_member(e, m, steps, &t)) == PLC_OK) e->cost[m] = t;
  }
  // 2. the batched launches' families, tiles and z chunk on the members' fields
  if (rc == PLC_OK && any_mixed) {
    std::vector<plc_ctx *> mixed;
    for (plc_ctx *c : e->members)
      if (c->mixed) mixed.push_back(c);
    for (plc_ctx *c : mixed) {
      const cudaError_t r = cudaStreamSynchronize(c->stream);
      if (r != cudaSuccess) rc = ens_cuda(e, r, "cudaStreamSynchronize");
    }
    if (rc == PLC_OK) {
      const cudaError_t r = plc::batch_autotune(mixed.data(), (int)mixed.size(), e->stream, &e->bplan);
      if (r != cudaSuccess) rc = ens_cuda(e, r, "batch_autotune");
      drop(e);
    }
  }
  // 3. every schedule on the ensemble graph; the fastest is kept
  int best = PLC_ENS_CONCURRENT;
  float best_t = -1.f;
  int best_chains = e->chains;
  bool best_pdl = e->bplan.pdl;
  const char *pdl_env = std::getenv("PLC_ENS_PDL");
  const int pdl_pin = pdl_env && pdl_env[0] == '1' ? 1 : pdl_env && pdl_env[0] == '0' ? 0 : -1;
  for (int s = 0; s < PLC_ENS_NUM_SCHEDULES && rc == PLC_OK; ++s) {
    if ((s == PLC_ENS_TWO_GROUPS && n < 2) || (s == PLC_ENS_BATCHED && !any_mixed)) {
      if (ms_per_scheme) ms_per_scheme[s] = -1.f;
      continue;
    }
    // the batched schedule: one chain of all the mixed-form members, or two
    // cost-balanced chains run concurrently; each with and without
    // programmatic dependent launch (unless PLC_ENS_PDL pins it)
    float t = -1.f;
    const int max_chains = s == PLC_ENS_BATCHED ? 2 : 1;
    const int pdl_lo = s == PLC_ENS_BATCHED && pdl_pin != 1 ? 0 : 1;
    const int pdl_hi = s == PLC_ENS_BATCHED && pdl_pin != 0 ? 1 : 0;
    for (int ch = 1; ch <= max_chains && rc == PLC_OK; ++ch) {
      for (int pd = s == PLC_ENS_BATCHED ? pdl_lo : 0; pd <= (s == PLC_ENS_BATCHED ? pdl_hi : 0);
           ++pd) {
        float tc = 0.f;
        if (s == PLC_ENS_BATCHED) {
          e->chains = ch;
          e->bplan.pdl = pd == 1;
        }
        if ((rc = apply_scheme(e, s)) != PLC_OK || (rc = time_launches(e, steps, &tc)) != PLC_OK)
          break;
        if (t < 0.f || tc < t) {
          t = tc;
          if (s == PLC_ENS_BATCHED) {
            best_chains = ch;
            best_pdl = pd == 1;
          }
        }
      }
      if (rc != PLC_OK) break;
    }
    if (rc != PLC_OK) break;
    t /= steps;
    if (ms_per_scheme) ms_per_scheme[s] = t;
    if (best_t < 0.f || t < best_t) {
      best_t = t;
      best = s;
    }
  }
  e->chains = best_chains;
  e->bplan.pdl = best_pdl;
  drop(e);
  if (rc == PLC_OK) rc = apply_scheme(e, best);
  const int rc2 = snapshot(e, snap, false);
  return rc != PLC_OK ? rc : rc2;
}

int plc_ensemble_set_batch_chains(plc_ensemble *e, int chains) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  if (chains < 1 || chains > 2) return ens_error(e, PLC_ERR_ARG, "chains must be 1 or 2");
  if (chains != e->chains) {
    e->chains = chains;
    drop(e);
  }
  return PLC_OK;
}

int plc_ensemble_set_batch_pdl(plc_ensemble *e, int on) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  if ((on != 0) != e->bplan.pdl) {
    e->bplan.pdl = on != 0;
    drop(e);
  }
  return PLC_OK;
}

int plc_ensemble_batch_pdl(const plc_ensemble *e, int *on) {
  if (!e || !on) return ens_error(nullptr, PLC_ERR_ARG, "null argument");
  *on = e->bplan.pdl ? 1 : 0;
  return PLC_OK;
}

int plc_ensemble_batch_choice(const plc_ensemble *e, int *chains, int *rk_kchunk,
                              int *rk_blocks_per_sm, int *fft_groups) {
  if (!e) return ens_error(nullptr, PLC_ERR_ARG, "null ensemble");
  if (chains) *chains = e->chains;
  if (rk_kchunk) *rk_kchunk = e->bplan.rk_kchunk;
  if (rk_blocks_per_sm) *rk_blocks_per_sm = e->bplan.rk_minb;
  if (fft_groups)
    for (int d = 0; d < 3; ++d) fft_groups[d] = (int)e->bplan.dir[d].size();
  return PLC_OK;
}

int plc_ensemble_partition(int n, const double *cost, int n_gpus, int *gpu_of) {
  if (n < 0 || n_gpus < 1 || (n > 0 && (!cost || !gpu_of)))
    return ens_error(nullptr, PLC_ERR_ARG, "bad argument");
  // longest processing time first: the costliest member to the least loaded GPU
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<double> load(n_gpus, 0.0);
  for (int m : order) {
    const int g = int(std::min_element(load.begin(), load.end()) - load.begin());
    gpu_of[m] = g;
    load[g] += cost[m];
  }
  return PLC_OK;
}

}  // extern "C"
