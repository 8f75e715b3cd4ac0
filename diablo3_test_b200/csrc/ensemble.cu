// Ensembles of independent channels stepped by CUDA graph launches, and the
// tile autotuner of the step transforms.
#include "internal.h"
#include "kernels_field.cuh"

// ==========================================================================
// Ensembles: independent members stepped by one CUDA graph launch per step.
// Each member's kernel chain is one branch of the graph (its own stream
// during capture), so small members run concurrently.  Kernel arguments hold
// the double-buffer pointers, so two graphs are kept, one per buffer parity.

struct MemberKey {
  int cur, cf_cur, les, generation;
  bool operator==(const MemberKey& o) const {
    return cur == o.cur && cf_cur == o.cf_cur && les == o.les && generation == o.generation;
  }
};

// One launch of the ensemble column step: the members of one rows-per-lane
// class R at one substep of one graph parity.  The member arguments are built
// on the host during capture and copied to the device after it.
struct EnsTable {
  int R = 0, ntask = 0;
  std::vector<int> members;        // indices into diablo_ensemble::m
  std::vector<FieldArgs> args;     // host copy, in member order
  std::vector<int> prefix;         // [nmem + 1] first task of each member
  FieldArgs* d_args = nullptr;
  int* d_prefix = nullptr;
  int* d_counter = nullptr;
};

struct diablo_ensemble {
  std::vector<diablo_ctx*> m;
  // DIABLO_ENSEMBLE_PERSISTENT: every member's column step of a substep in
  // one persistent launch per rows-per-lane class; DIABLO_ENSEMBLE_BRANCHES:
  // each member's whole step on its own graph branch
  int mode = DIABLO_ENSEMBLE_PERSISTENT;
  std::vector<EnsTable> tables[2][3];   // [graph parity][substep]
  // per rows-per-lane class (R = 3..9): the stream its column launches are
  // captured on and the event the class's members wait on
  cudaStream_t cstream[10] = {};
  cudaEvent_t cevent[10] = {};
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  std::vector<MemberKey> key[2];
  std::vector<long long> nlaunch[2];
  int last_cuda = 0;
};

MemberKey member_key(const diablo_ctx* c) {
  return MemberKey{c->cur, c->cf_cur, les_active(c), c->generation};
}

// Everything a step allocates on first use, so that capture allocates nothing.
int prepare_member(diablo_ctx* ctx) {
  int rc;
  if ((rc = ensure_scratch(ctx))) return rc;
  if (les_active(ctx)) {
    if ((rc = ensure_les(ctx))) return rc;
    const int m = ctx->p.les_model_type;
    if ((m == 4 || m == 5) && (rc = ensure_amd(ctx))) return rc;
    if (m == 2 && (rc = ensure_dyn(ctx))) return rc;
  }
  return 0;
}

int one_step(diablo_ctx* ctx) {
  ctx->time_step += 1;
  for (int rk = 1; rk <= 3; ++rk) {
    int rc = substep(ctx, rk);
    if (rc) return rc;
  }
  ctx->time += ctx->delta_t;
  return 0;
}

#define ECK(call)                                 \
  do {                                            \
    cudaError_t e__ = (call);                     \
    if (e__ != cudaSuccess) {                     \
      e->last_cuda = (int)e__;                    \
      return DIABLO_ERR_CUDA;                     \
    }                                             \
  } while (0)

// Capture one step of every member into exec[w], from the members' current
// host state; the host state is advanced as the step would advance it.
int capture(diablo_ensemble* e, int w) {
  const int n = (int)e->m.size();
  std::vector<cudaStream_t> saved(n);
  std::vector<int> prof(n);
  e->key[w].resize(n);
  e->nlaunch[w].resize(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    saved[i] = c->stream;
    prof[i] = c->profiling;
    c->profiling = 0;
    c->stream = e->streams[i];
    e->key[w][i] = member_key(c);
  }
  cudaGraph_t graph = nullptr;
  int rc = 0;
  cudaError_t ce = cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    cudaEventRecord(e->fork, e->origin);
    for (int i = 0; i < n && !rc; ++i) {
      diablo_ctx* c = e->m[i];
      cudaStreamWaitEvent(e->streams[i], e->fork, 0);
      const long long l0 = c->launches;
      rc = one_step(c);
      e->nlaunch[w][i] = c->launches - l0;
      cudaEventRecord(e->joins[i], e->streams[i]);
      cudaStreamWaitEvent(e->origin, e->joins[i], 0);
    }
    ce = cudaStreamEndCapture(e->origin, &graph);
  }
  for (int i = 0; i < n; ++i) {
    e->m[i]->stream = saved[i];
    e->m[i]->profiling = prof[i];
  }
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc;
  }
  ECK(ce);
  if (e->exec[w]) { cudaGraphExecDestroy(e->exec[w]); e->exec[w] = nullptr; }
  ce = cudaGraphInstantiate(&e->exec[w], graph, 0);
  cudaGraphDestroy(graph);
  ECK(ce);
  return 0;
}

// Whether every member's substep takes the field-split column step that the
// ensemble kernel runs: DNS (LES gate never opening), no 'Front' forcing,
// the default column path, and 3..9 rows per lane.
bool persistent_ok(const diablo_ensemble* e) {
  for (const diablo_ctx* c : e->m) {
    if (c->p.use_les || (c->p.flavor_front && c->ro_inv != 0.0)) return false;
    if (!(c->use_general_solver == 0 || c->use_general_solver == 3)) return false;
    const int R = rows_per_lane(c->nyp2);
    if (R < 3 || R > 9 || column_step_ens_resident(R) <= 0) return false;
  }
  return true;
}

void free_tables(diablo_ensemble* e, int w) {
  for (int rk = 0; rk < 3; ++rk) {
    for (EnsTable& t : e->tables[w][rk]) {
      if (t.d_args) cudaFree(t.d_args);
      if (t.d_prefix) cudaFree(t.d_prefix);
      if (t.d_counter) cudaFree(t.d_counter);
    }
    e->tables[w][rk].clear();
  }
}

// Capture one step of every member into exec[w] with the column steps of
// each substep launched together: per substep, each member's transforms and
// nonlinear terms on its own branch, then (after all branches) one
// k_column_step_ens launch per rows-per-lane class, then the next substep's
// branches.  The host state is advanced as the step would advance it.
int capture_persistent(diablo_ensemble* e, int w) {
  const int n = (int)e->m.size();
  for (diablo_ctx* c : e->m) {
    const int R = rows_per_lane(c->nyp2);
    if (!e->cstream[R] && (cudaStreamCreateWithFlags(&e->cstream[R], cudaStreamNonBlocking) != cudaSuccess ||
                           cudaEventCreateWithFlags(&e->cevent[R], cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      return DIABLO_ERR_CUDA;
    }
  }
  // classes and their device tables (allocated before capture begins)
  free_tables(e, w);
  for (int rk = 0; rk < 3; ++rk) {
    std::vector<EnsTable>& tb = e->tables[w][rk];
    for (int i = 0; i < n; ++i) {
      const int R = rows_per_lane(e->m[i]->nyp2);
      EnsTable* t = nullptr;
      for (EnsTable& x : tb) if (x.R == R) t = &x;
      if (!t) { tb.emplace_back(); t = &tb.back(); t->R = R; }
      t->members.push_back(i);
    }
    for (EnsTable& t : tb) {
      const size_t k = t.members.size();
      t.args.assign(k, FieldArgs{});
      t.prefix.assign(k + 1, 0);
      if (cudaMalloc((void**)&t.d_args, k * sizeof(FieldArgs)) != cudaSuccess ||
          cudaMalloc((void**)&t.d_prefix, (k + 1) * sizeof(int)) != cudaSuccess ||
          cudaMalloc((void**)&t.d_counter, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        free_tables(e, w);
        return DIABLO_ERR_NOMEM;
      }
    }
  }
  std::vector<cudaStream_t> saved(n);
  std::vector<int> prof(n);
  e->key[w].resize(n);
  e->nlaunch[w].assign(n, 0);
  std::vector<long long> l0(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    saved[i] = c->stream;
    prof[i] = c->profiling;
    c->profiling = 0;
    c->stream = e->streams[i];
    e->key[w][i] = member_key(c);
    l0[i] = c->launches;
  }
  cudaGraph_t graph = nullptr;
  int rc = 0;
  cudaError_t ce = cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    cudaEventRecord(e->fork, e->origin);
    for (int rk = 1; rk <= 3 && !rc; ++rk) {
      std::vector<EnsTable>& tb = e->tables[w][rk - 1];
      for (EnsTable& t : tb) {
        for (size_t k = 0; k < t.members.size() && !rc; ++k) {
          diablo_ctx* c = e->m[t.members[k]];
          // the step's start, or this class's column step of the substep before
          cudaStreamWaitEvent(c->stream, rk == 1 ? e->fork : e->cevent[t.R], 0);
          if (rk == 1) c->time_step += 1;
          c->defer_col = &t.args[k];
          c->defer_filled = 0;
          rc = substep(c, rk);
          c->defer_col = nullptr;
          if (!rc && !c->defer_filled) rc = DIABLO_ERR_UNSUPPORTED;
          if (rk == 3) c->time += c->delta_t;
          cudaEventRecord(e->joins[t.members[k]], c->stream);
          cudaStreamWaitEvent(e->cstream[t.R], e->joins[t.members[k]], 0);
        }
      }
      for (EnsTable& t : tb) {
        if (rc) break;
        const int res = column_step_ens_resident(t.R);
        int tot = 0;
        for (size_t k = 0; k < t.members.size(); ++k) {
          FieldArgs& F = t.args[k];
          const int ngroup = (F.s.ncol + FS_COLS - 1) / FS_COLS;
          F.lag = std::max(1, res / F.nf);
          t.prefix[k] = tot;
          tot += ngroup * (F.nf + 1);
        }
        t.prefix[t.members.size()] = tot;
        t.ntask = tot;
        EnsColArgs E;
        E.mem = t.d_args;
        E.prefix = t.d_prefix;
        E.counter = t.d_counter;
        E.nmem = (int)t.members.size();
        E.tsz = 32 * t.R * FS_COLS;
        rc = launch_column_step_ens(E, t.R, tot, e->cstream[t.R]);
        e->nlaunch[w][t.members[0]] += 2;
        cudaEventRecord(e->cevent[t.R], e->cstream[t.R]);
      }
    }
    // the step ends when every class's last column step has
    for (EnsTable& t : e->tables[w][2]) cudaStreamWaitEvent(e->origin, e->cevent[t.R], 0);
    ce = cudaStreamEndCapture(e->origin, &graph);
  }
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    e->nlaunch[w][i] += c->launches - l0[i];
    c->launches = l0[i];
    c->stream = saved[i];
    c->profiling = prof[i];
  }
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc;
  }
  ECK(ce);
  // the member tables the graph's kernels read
  for (int rk = 0; rk < 3; ++rk)
    for (EnsTable& t : e->tables[w][rk]) {
      ECK(cudaMemcpy(t.d_args, t.args.data(), t.args.size() * sizeof(FieldArgs), cudaMemcpyHostToDevice));
      ECK(cudaMemcpy(t.d_prefix, t.prefix.data(), t.prefix.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
  if (e->exec[w]) { cudaGraphExecDestroy(e->exec[w]); e->exec[w] = nullptr; }
  ce = cudaGraphInstantiate(&e->exec[w], graph, 0);
  cudaGraphDestroy(graph);
  ECK(ce);
  return 0;
}

// (Re)capture both graphs from the members' current state, leaving the
// members' host state as it was.
int capture_both(diablo_ensemble* e) {
  const int n = (int)e->m.size();
  struct Saved { double time; int time_step, cur, cf_cur; double wtt; };
  std::vector<Saved> sv(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    int rc = prepare_member(c);
    if (rc) return rc;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return DIABLO_ERR_CUDA;
    sv[i] = Saved{c->time, c->time_step, c->cur, c->cf_cur, c->w_top_transient};
  }
  const bool pers = e->mode == DIABLO_ENSEMBLE_PERSISTENT;
  int rc = pers ? capture_persistent(e, 0) : capture(e, 0);
  if (!rc) rc = pers ? capture_persistent(e, 1) : capture(e, 1);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    c->time = sv[i].time; c->time_step = sv[i].time_step;
    c->cur = sv[i].cur; c->cf_cur = sv[i].cf_cur; c->w_top_transient = sv[i].wtt;
  }
  return rc;
}

extern "C" {

diablo_ensemble* diablo_ensemble_create(diablo_ctx* const* members, int n, int* status) {
  int st = 0;
  diablo_ensemble* e = nullptr;
  if (!members || n <= 0) st = DIABLO_ERR_ARG;
  for (int i = 0; i < n && !st; ++i) {
    const diablo_ctx* c = members[i];
    if (!c) { st = DIABLO_ERR_ARG; break; }
    for (int k = 0; k < i; ++k)
      if (members[k] == c) st = DIABLO_ERR_ARG;
    // kernel arguments that change every step cannot be replayed from a graph
    if (c->p.variable_dt || c->p.f_type == 2 || (c->p.f_type == 4 && c->p.w_bc_ymax != 0))
      st = DIABLO_ERR_UNSUPPORTED;
    for (int q = 0; q < c->nth; ++q)
      if (c->p.filter_th[q]) st = DIABLO_ERR_UNSUPPORTED;   // filtered on some steps only
  }
  if (!st) {
    e = new diablo_ensemble();
    e->m.assign(members, members + n);
    bool ok = cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
    e->streams.assign(n, nullptr);
    e->joins.assign(n, nullptr);
    for (int i = 0; i < n && ok; ++i)
      ok = cudaStreamCreateWithFlags(&e->streams[i], cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&e->joins[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) { st = DIABLO_ERR_CUDA; diablo_ensemble_destroy(e); e = nullptr; }
    else e->mode = persistent_ok(e) ? DIABLO_ENSEMBLE_PERSISTENT : DIABLO_ENSEMBLE_BRANCHES;
  }
  if (status) *status = st;
  return e;
}

int diablo_ensemble_step(diablo_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return DIABLO_ERR_ARG;
  const int n = (int)e->m.size();
  for (int s = 0; s < nsteps; ++s) {
    // the graph captured for this parity must match every member's state
    int w = -1;
    for (int k = 0; k < 2 && w < 0; ++k) {
      if (!e->exec[k] || (int)e->key[k].size() != n) continue;
      bool ok = true;
      for (int i = 0; i < n && ok; ++i) ok = member_key(e->m[i]) == e->key[k][i];
      if (ok) w = k;
    }
    if (w < 0) {
      int rc = capture_both(e);
      if (rc) return rc;
      w = 0;
    }
    // order the graph after each member's earlier work on its own stream
    for (int i = 0; i < n; ++i) {
      ECK(cudaEventRecord(e->joins[i], e->m[i]->stream));
      ECK(cudaStreamWaitEvent(e->origin, e->joins[i], 0));
    }
    ECK(cudaGraphLaunch(e->exec[w], e->origin));
    ECK(cudaEventRecord(e->fork, e->origin));
    for (int i = 0; i < n; ++i) {
      diablo_ctx* c = e->m[i];
      ECK(cudaStreamWaitEvent(c->stream, e->fork, 0));
      c->time_step += 1;
      c->time += c->delta_t;
      c->cur ^= 1;                 // three substeps flip the state buffer
      c->launches += e->nlaunch[w][i];
    }
  }
  return 0;
}

void* diablo_ensemble_stream(diablo_ensemble* e) { return e ? (void*)e->origin : nullptr; }

int diablo_ensemble_set_mode(diablo_ensemble* e, int mode) {
  if (!e || (mode != DIABLO_ENSEMBLE_BRANCHES && mode != DIABLO_ENSEMBLE_PERSISTENT)) return DIABLO_ERR_ARG;
  if (mode == DIABLO_ENSEMBLE_PERSISTENT && !persistent_ok(e)) return DIABLO_ERR_UNSUPPORTED;
  if (mode == e->mode) return 0;
  ECK(cudaStreamSynchronize(e->origin));
  for (int k = 0; k < 2; ++k) {
    if (e->exec[k]) { cudaGraphExecDestroy(e->exec[k]); e->exec[k] = nullptr; }
    e->key[k].clear();
  }
  e->mode = mode;
  return 0;
}

int diablo_ensemble_mode(const diablo_ensemble* e) { return e ? e->mode : DIABLO_ERR_ARG; }

int diablo_ensemble_synchronize(diablo_ensemble* e) {
  if (!e) return DIABLO_ERR_ARG;
  ECK(cudaStreamSynchronize(e->origin));
  for (diablo_ctx* c : e->m) ECK(cudaStreamSynchronize(c->stream));
  ECK(cudaGetLastError());
  int rc = 0;
  for (diablo_ctx* c : e->m) {   // a member's column-step wait that gave up
    const int r = sched_status(c);
    if (r && !rc) rc = r;
  }
  return rc;
}

int diablo_ensemble_destroy(diablo_ensemble* e) {
  if (!e) return DIABLO_ERR_ARG;
  if (e->origin) cudaStreamSynchronize(e->origin);
  for (int k = 0; k < 2; ++k)
    if (e->exec[k]) cudaGraphExecDestroy(e->exec[k]);
  for (int k = 0; k < 2; ++k) free_tables(e, k);
  for (int r = 0; r < 10; ++r) {
    if (e->cstream[r]) cudaStreamDestroy(e->cstream[r]);
    if (e->cevent[r]) cudaEventDestroy(e->cevent[r]);
  }
  for (cudaStream_t s : e->streams)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t v : e->joins)
    if (v) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->origin) cudaStreamDestroy(e->origin);
  delete e;
  return 0;
}

}  // extern "C"

// ==========================================================================
// Autotuner: the tile shapes of the four step transforms (sequences per
// block of the z kernels, rows per block of the x kernels) are timed on the
// context's own scratch for its grid and precision, and the fastest kept.
// Results are cached per (grid, fields, precision) for the process.

#include <map>
#include <mutex>
#include <tuple>

static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int, int>, std::array<int, 4>> g_tune_cache;

extern "C" {

int diablo_tiles(diablo_ctx* ctx, int* tiles) {
  if (!ctx || !tiles) return DIABLO_ERR_ARG;
  for (int q = 0; q < 4; ++q) tiles[q] = ctx->tune[q];
  return 0;
}

int diablo_autotune(diablo_ctx* ctx, int* tiles) {
  if (!ctx) return DIABLO_ERR_ARG;
  int rc;
  if (les_active(ctx)) return DIABLO_ERR_UNSUPPORTED;
  if ((rc = ensure_scratch(ctx))) return rc;
  const auto key = std::make_tuple(ctx->nx, ctx->ny, ctx->nz, ctx->nf, ctx->precision);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      for (int q = 0; q < 4; ++q) ctx->tune[q] = it->second[q];
      ctx->generation++;
      if (tiles) for (int q = 0; q < 4; ++q) tiles[q] = ctx->tune[q];
      return 0;
    }
  }
  const bool fp32 = ctx->precision != DIABLO_FP64;
  SolveArgs sa;
  fill_solve_args(ctx, sa, 1);
  const bool mean_split = fp32 && !sa.front && ctx->use_general_solver != 1;
  int cand[4][3], nc[4];
  for (int k = 0; k < 4; ++k) {
    nc[k] = fft_tile_candidates(k, (k == 0 || k == 3) ? ctx->nz : ctx->M, fp32, cand[k]);
    if (nc[k] <= 0) return DIABLO_ERR_SIZE;
  }
  const int slot[4] = {K_ZINV, K_XINV, K_XFWD_NL, K_ZFWD_NL};
  double best[4] = {1e300, 1e300, 1e300, 1e300};
  int pick[4] = {0, 0, 0, 0};
  const int saved_prof = ctx->profiling;
  auto run = [&]() -> int {
    return fp32 ? substep_spectral<float>(ctx, mean_split ? 0x1u : 0u) : substep_spectral<double>(ctx, 0u);
  };
  for (int i = 0; i < 3; ++i) {
    for (int k = 0; k < 4; ++k) ctx->tune[k] = cand[k][i < nc[k] ? i : nc[k] - 1];
    ctx->profiling = 0;
    if ((rc = run())) { ctx->profiling = saved_prof; return rc; }
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    ctx->profiling = 1;
    for (int sl = 0; sl < K_NSLOTS; ++sl) { ctx->slot_ms[sl] = 0.0; ctx->slot_n[sl] = 0; }
    for (int r = 0; r < 3 && !rc; ++r) rc = run();
    if (rc) { ctx->profiling = saved_prof; return rc; }
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    for (int k = 0; k < 4; ++k) {
      if (i >= nc[k]) continue;
      const double t = ctx->slot_ms[slot[k]];
      if (t < best[k]) { best[k] = t; pick[k] = cand[k][i]; }
    }
  }
  for (int sl = 0; sl < K_NSLOTS; ++sl) { ctx->slot_ms[sl] = 0.0; ctx->slot_n[sl] = 0; }
  ctx->profiling = saved_prof;
  for (int k = 0; k < 4; ++k) ctx->tune[k] = pick[k];
  ctx->generation++;
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_cache[key] = {pick[0], pick[1], pick[2], pick[3]};
  }
  if (tiles) for (int q = 0; q < 4; ++q) tiles[q] = pick[q];
  return 0;
}

}  // extern "C"

// ==========================================================================
// Ensemble autotuner: coordinate descent over the transform tiles of each
// group of same-size members, scored by the time of the ensemble's own graph
// (the members' kernels run concurrently there, so isolated kernel times are
// not the objective).  Member states are restored afterwards.

extern "C" {

int diablo_ensemble_autotune(diablo_ensemble* e, int steps_per_trial) {
  if (!e || steps_per_trial <= 0) return DIABLO_ERR_ARG;
  const int n = (int)e->m.size();
  int rc;
  // snapshot every member (state fields, counters, tiles)
  struct Snap { std::vector<double2*> f; double time; int step, cur, cf_cur; int tune[4]; };
  std::vector<Snap> snap(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    if ((rc = ensure_scratch(c))) return rc;
    if (les_active(c)) return DIABLO_ERR_UNSUPPORTED;
    const size_t fe = four_elems(c) * sizeof(double2);
    snap[i].f.assign(4 + c->nth, nullptr);
    for (int q = 0; q < 4 + c->nth; ++q) {
      if ((rc = dev_alloc(c, (void**)&snap[i].f[q], fe))) return rc;
      if (cudaMemcpyAsync(snap[i].f[q], c->st[c->cur][q], fe, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        return DIABLO_ERR_CUDA;
    }
    snap[i].time = c->time; snap[i].step = c->time_step; snap[i].cur = c->cur; snap[i].cf_cur = c->cf_cur;
    for (int q = 0; q < 4; ++q) snap[i].tune[q] = c->tune[q];
  }
  // groups of members sharing a tile configuration
  std::vector<std::vector<int>> groups;
  std::vector<std::tuple<int, int, int, int, int>> gkey;
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    auto k = std::make_tuple(c->nx, c->ny, c->nz, c->nf, c->precision);
    size_t g = 0;
    while (g < gkey.size() && gkey[g] != k) ++g;
    if (g == gkey.size()) { gkey.push_back(k); groups.emplace_back(); }
    groups[g].push_back(i);
  }
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto trial = [&](float* ms) -> int {
    int r = diablo_ensemble_step(e, 1);      // captures if needed, warms
    if (r) return r;
    ECK(cudaEventRecord(t0, e->origin));
    if ((r = diablo_ensemble_step(e, steps_per_trial))) return r;
    ECK(cudaEventRecord(t1, e->origin));
    ECK(cudaEventSynchronize(t1));
    ECK(cudaEventElapsedTime(ms, t0, t1));
    return 0;
  };
  float best = 0.f;
  rc = trial(&best);
  for (size_t g = 0; g < groups.size() && !rc; ++g) {
    diablo_ctx* c0 = e->m[groups[g][0]];
    const bool fp32 = c0->precision != DIABLO_FP64;
    for (int k = 0; k < 4 && !rc; ++k) {
      int cand[3];
      const int nc = fft_tile_candidates(k, (k == 0 || k == 3) ? c0->nz : c0->M, fp32, cand);
      const int keep = c0->tune[k];
      int pick = keep;
      for (int ci = 0; ci < nc && !rc; ++ci) {
        if (cand[ci] == keep || (keep == 0 && ci == 0)) continue;   // the current choice is already scored
        for (int i : groups[g]) { e->m[i]->tune[k] = cand[ci]; e->m[i]->generation++; }
        float ms = 0.f;
        if ((rc = trial(&ms))) break;
        if (ms < best) { best = ms; pick = cand[ci]; }
      }
      for (int i : groups[g]) { e->m[i]->tune[k] = pick; e->m[i]->generation++; }
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  // restore the members' states (the tiles found are kept)
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = rc ? rc : DIABLO_ERR_CUDA;
    c->cur = snap[i].cur; c->cf_cur = snap[i].cf_cur; c->time = snap[i].time; c->time_step = snap[i].step;
    const size_t fe = four_elems(c) * sizeof(double2);
    for (int q = 0; q < 4 + c->nth; ++q) {
      cudaMemcpyAsync(c->st[c->cur][q], snap[i].f[q], fe, cudaMemcpyDeviceToDevice, c->stream);
      cudaStreamSynchronize(c->stream);
      for (size_t a = 0; a < c->allocs.size(); ++a)
        if (c->allocs[a] == snap[i].f[q]) { c->allocs.erase(c->allocs.begin() + a); break; }
      cudaFree(snap[i].f[q]);
    }
    if (rc) for (int q = 0; q < 4; ++q) c->tune[q] = snap[i].tune[q];
    c->generation++;
  }
  return rc;
}

}  // extern "C"

