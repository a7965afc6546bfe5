// C ABI of the library and the skeleton runner.
//
// Skeleton semantics (pcalg "stable", as replayed by the reference in
// fastkpc/src/full_cuda_ci_one_call.cpp:5229-5579 over the plan of
// fastkpc/src/skeleton_task_scheduler.cpp:70-132):
//  * level plan: for each edge x < y of the level-start adjacency, the x-side
//    tasks (S over combinations of adj(x)\{y} of size ``level``, in
//    lexicographic order) then the y-side tasks; a side's first task "opens
//    the next level" when the side has more than ``level`` neighbours;
//  * per edge the tasks count in plan order up to and including the first
//    deleting one (p >= alpha); pMax keeps the max p per edge, the deleting
//    S becomes the sepset, deletions apply at level end; the run stops after
//    a level where no counted task opens the next level, or past m.max.
// The batched form evaluates every planned task of a level in one batch
// (tests are independent given the level-start graph) and then replays; the
// counted tests, graph, sepsets and trace are those of the sequential order.
// Permutation methods draw their tables from one R-compatible stream in
// pcalg order (x, y, S lexicographic) over the counted tests, so they run one
// test at a time in that order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fastkpc_b200.h"
#include "orient.h"
#include "runtime.h"

namespace {

thread_local std::string g_last_error;

}  // namespace

namespace fkpc {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace fkpc

namespace {

// One engine per device, each behind its own mutex: calls on different
// devices run concurrently (one host thread per GPU), calls on one device
// are serialised.
struct EngineSlot {
  std::mutex mu;
  std::unique_ptr<fkpc::Engine> eng;
  uint64_t session = 0;  // load_id of the data fkpc_session_load left loaded (0: none)
};
std::mutex g_slots_mu;
std::map<int, std::unique_ptr<EngineSlot>> g_slots;

EngineSlot& slot_for(int device) {
  std::lock_guard<std::mutex> lock(g_slots_mu);
  auto& p = g_slots[device];
  if (!p) p.reset(new EngineSlot());
  return *p;
}

std::mutex& device_mutex(int device) { return slot_for(device).mu; }

// The device's engine; call with device_mutex(device) held.
fkpc::Engine& engine_for(int device) {
  EngineSlot& s = slot_for(device);
  if (!s.eng) s.eng.reset(new fkpc::Engine(device));
  return *s.eng;
}

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return FKPC_OK;
  } catch (const fkpc::Error& e) {
    return fail(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return fail(FKPC_STATUS_ALLOCATION, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(FKPC_STATUS_INVALID_ARGUMENT, e.what());
  }
}

void validate_options(const fkpc_options& o, int n, int p) {
  using fkpc::Error;
  if (!(std::isfinite(o.alpha) && o.alpha > 0.0 && o.alpha < 1.0))
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "alpha must lie in (0, 1)");
  if (o.index != 1.0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "index must be 1 (legacy dCov semantics)");
  if (o.num_col < 1 || o.num_col > 64 || o.num_col >= n)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "numCol must lie in [1, min(64, n - 1)]");
  if (o.ci_method < FKPC_DCC_GAMMA || o.ci_method > FKPC_HSIC_PERM)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "unknown CI method");
  if (!(std::isfinite(o.hsic_sig) && o.hsic_sig > 0.0))
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "HSIC sig must be positive and finite");
  if (o.ci_method == FKPC_DCC_PERM || o.ci_method == FKPC_HSIC_PERM) {
    if (!o.has_seed) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation methods require a seed");
    if (o.permutation_replicates < 1 || o.permutation_replicates > 10000)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation replicates must lie in [1, 10000]");
    if (n > 32768) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation methods support n <= 32768");
  }
  if (o.mode != FKPC_MODE_BATCHED && o.mode != FKPC_MODE_PLAIN)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "unknown execution mode");
  if (o.selection != FKPC_SELECT_MAGIC && o.selection != FKPC_SELECT_GN_NEWTON)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "selection must be FKPC_SELECT_MAGIC or FKPC_SELECT_GN_NEWTON");
  if (p < 2 || n <= 5) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "need n > 5 and p >= 2");
  if (o.strict) {
    // the qualified envelope of fastkpc/src/full_cuda_ci_one_call.cpp:5052-5087
    if (std::fabs(o.alpha - 0.1) > 1e-15) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "strict mode requires alpha = 0.1");
    if (o.num_col != 35) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "strict mode requires numCol = 35");
    if (p > 64) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "strict mode requires 2 <= p <= 64");
  }
}

struct Task {
  int edge_x, edge_y, x, y;
  std::vector<int> S;
  bool opens;
};

std::vector<Task> make_layer_plan(const std::vector<int>& adj, int p, int level) {
  std::vector<Task> tasks;
  auto nbrs = [&](int v, int excl) {
    std::vector<int> out;
    for (int i = 0; i < p; ++i)
      if (i != excl && adj[i + static_cast<size_t>(p) * v]) out.push_back(i);
    return out;
  };
  for (int x = 0; x < p - 1; ++x)
    for (int y = x + 1; y < p; ++y) {
      if (!adj[x + static_cast<size_t>(p) * y]) continue;
      for (int side = 0; side < 2; ++side) {
        const int a = side == 0 ? x : y, b = side == 0 ? y : x;
        const std::vector<int> nb = nbrs(a, b);
        if (static_cast<int>(nb.size()) < level) continue;
        std::vector<int> idx(level);
        for (int i = 0; i < level; ++i) idx[i] = i;
        bool first = true;
        for (;;) {
          Task t;
          t.edge_x = x;
          t.edge_y = y;
          t.x = a;
          t.y = b;
          for (int i = 0; i < level; ++i) t.S.push_back(nb[idx[i]]);
          t.opens = first && static_cast<int>(nb.size()) > level;
          first = false;
          tasks.push_back(std::move(t));
          int i = level - 1;
          while (i >= 0 && idx[i] == static_cast<int>(nb.size()) - level + i) --i;
          if (i < 0) break;
          ++idx[i];
          for (int j = i + 1; j < level; ++j) idx[j] = idx[j - 1] + 1;
        }
      }
    }
  return tasks;
}

struct Run {
  int n = 0, p = 0;
  std::vector<int> adj;
  std::vector<double> pmax;
  std::map<std::pair<int, int>, std::vector<int>> sepsets;
  std::vector<int> n_edgetests;
  std::vector<fkpc_trace_row> trace;
  std::vector<int> trace_s;
  fkpc_stage_stats stats{};
};

void add_stats(fkpc_stage_stats* acc, const fkpc_stage_stats& s) {
  acc->setup_ms += s.setup_ms;
  acc->upload_ms += s.upload_ms;
  acc->fit_ms += s.fit_ms;
  acc->statistic_ms += s.statistic_ms;
  acc->refine_ms += s.refine_ms;
  acc->download_ms += s.download_ms;
  acc->designs += s.designs;
  acc->targets += s.targets;
  acc->pairs += s.pairs;
  acc->guarded += s.guarded;
  acc->kernel_launches += s.kernel_launches;
  acc->h2d_bytes += s.h2d_bytes;
  acc->d2h_bytes += s.d2h_bytes;
  acc->fit_evaluations += s.fit_evaluations;
  acc->fit_flops += s.fit_flops;
  acc->statistic_flops += s.statistic_flops;
  acc->fit_iterations += s.fit_iterations;
  acc->lowrank_components += s.lowrank_components;
  acc->lowrank_steps_max = std::max(acc->lowrank_steps_max, s.lowrank_steps_max);
  acc->lowrank_steps_mean = s.lowrank_steps_mean;
  acc->device_ms += s.device_ms;
  acc->designs_built += s.designs_built;
  acc->smooths_built += s.smooths_built;
  acc->plan_ms += s.plan_ms;
  acc->tprs_host_ms += s.tprs_host_ms;
  acc->design_host_ms += s.design_host_ms;
  acc->smooth_wait_ms += s.smooth_wait_ms;
  acc->late_wait_ms += s.late_wait_ms;
  acc->prefit_device_ms += s.prefit_device_ms;
}

// Evaluate ``tests`` on the engine in chunks; records in test order.
void evaluate(fkpc::Engine& eng, const std::vector<fkpc::Test>& tests, const fkpc_options& opt, fkpc::RStream* rs,
              std::vector<fkpc_ci_record>* out, fkpc_stage_stats* acc) {
  out->resize(tests.size());
  size_t chunk = opt.mode == FKPC_MODE_PLAIN ? 1 : 16384;
  if (opt.ci_method == FKPC_DCC_PERM || opt.ci_method == FKPC_HSIC_PERM) {
    // permutation tables are R x n int32 per test: keep each chunk's table
    // near 1 GiB (tests stay in order, so the seeded stream is consumed as in
    // one pass)
    const size_t per_test = static_cast<size_t>(opt.permutation_replicates) * static_cast<size_t>(eng.n()) * sizeof(int);
    chunk = std::min(chunk, std::max<size_t>(1, (static_cast<size_t>(1) << 30) / std::max<size_t>(1, per_test)));
  }
  for (size_t b = 0; b < tests.size(); b += chunk) {
    const size_t e = std::min(tests.size(), b + chunk);
    std::vector<fkpc::Test> part(tests.begin() + b, tests.begin() + e);
    fkpc_stage_stats st{};
    const bool perm = opt.ci_method == FKPC_DCC_PERM || opt.ci_method == FKPC_HSIC_PERM;
    if (opt.mode == FKPC_MODE_PLAIN || (opt.level_graph && !perm)) {
      eng.prepare(part, opt, rs);  // set-up, then the captured launch sequence
      eng.execute();
    } else {
      eng.run_batch(part, opt, rs);
    }
    eng.collect(out->data() + b, &st);
    add_stats(acc, st);
  }
}

void skeleton(const double* data, int n, int p, const fkpc_options& opt, Run* run,
              fkpc_level_evaluator evaluator = nullptr, void* user = nullptr) {
  fkpc::Engine* engp = nullptr;
  if (!evaluator) {
    engp = &engine_for(opt.device);
    engp->load(data, n, p);
  }
  const int m_max = opt.max_conditioning_size < 0 ? p - 2 : std::min(opt.max_conditioning_size, p - 2);
  const bool perm = opt.ci_method == FKPC_DCC_PERM || opt.ci_method == FKPC_HSIC_PERM;
  std::unique_ptr<fkpc::RStream> rs;
  if (perm) rs.reset(new fkpc::RStream(opt.seed));
  run->n = n;
  run->p = p;
  run->adj.assign(static_cast<size_t>(p) * p, 1);
  for (int i = 0; i < p; ++i) run->adj[i + static_cast<size_t>(p) * i] = 0;
  run->pmax.assign(static_cast<size_t>(p) * p, -INFINITY);
  for (int level = 0; level <= m_max; ++level) {
    std::vector<Task> plan = make_layer_plan(run->adj, p, level);
    std::map<std::pair<int, int>, std::vector<int>> by_edge;
    for (size_t i = 0; i < plan.size(); ++i) by_edge[{plan[i].edge_x, plan[i].edge_y}].push_back(static_cast<int>(i));
    std::vector<double> pv(plan.size(), NAN), pe(plan.size(), NAN);
    std::vector<unsigned> fl(plan.size(), 0u);
    std::vector<char> counted(plan.size(), 0);
    auto to_test = [&](const Task& t) { return fkpc::Test{t.x, t.y, t.S}; };
    if (perm && opt.mode != FKPC_MODE_PLAIN) {
      if (evaluator) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "the level evaluator serves the batched gamma methods");
      // Permutation methods draw their permutations from one seeded stream in
      // pcalg order (x, y, S), and an edge's remaining tests are skipped once
      // it is deleted.  Speculative windows: the next `window` tests of that
      // order, as if no edge were deleted, are evaluated as one batch (the
      // stream consumed test by test in window order).  Results are accepted
      // in order up to the first test that an accepted deletion skips; the
      // stream is then reset to its state after the last accepted test, and
      // the next window starts there.  Outcome and stream use are those of
      // the one-test-at-a-time order.
      std::map<std::pair<int, int>, size_t> pos;
      for (auto& kv : by_edge) pos[kv.first] = 0;
      auto pick = [&](const std::map<std::pair<int, int>, size_t>& at) {
        int best = -1;
        for (auto& kv : by_edge) {
          const size_t k = at.at(kv.first);
          if (k >= kv.second.size()) continue;
          const int cand = kv.second[k];
          if (best < 0) {
            best = cand;
            continue;
          }
          const Task& a = plan[cand];
          const Task& b = plan[best];
          if (a.x != b.x ? a.x < b.x : (a.y != b.y ? a.y < b.y : a.S < b.S)) best = cand;
        }
        return best;
      };
      size_t window = 32;
      std::vector<int> seq;
      for (;;) {
        seq.clear();
        auto at = pos;
        while (seq.size() < window) {
          const int b = pick(at);
          if (b < 0) break;
          seq.push_back(b);
          ++at[{plan[b].edge_x, plan[b].edge_y}];
        }
        if (seq.empty()) break;
        std::vector<fkpc::Test> tests;
        tests.reserve(seq.size());
        for (int b : seq) tests.push_back(to_test(plan[b]));
        std::vector<fkpc::RStream> snaps;
        std::vector<fkpc_ci_record> rec;
        engp->set_stream_snapshots(&snaps);
        try {
          evaluate(*engp, tests, opt, rs.get(), &rec, &run->stats);
        } catch (...) {
          engp->set_stream_snapshots(nullptr);
          throw;
        }
        engp->set_stream_snapshots(nullptr);
        if (snaps.size() != seq.size()) throw fkpc::Error(FKPC_STATUS_NUMERIC, "permutation stream snapshots incomplete");
        size_t limit = seq.size(), i = 0;
        for (; i < limit; ++i) {
          const int b = seq[i];
          pv[b] = rec[i].p_value;
          pe[b] = rec[i].p_exact;
          fl[b] = rec[i].flags;
          counted[b] = 1;
          const std::pair<int, int> key{plan[b].edge_x, plan[b].edge_y};
          if (rec[i].p_value >= opt.alpha) {
            pos[key] = by_edge[key].size();
            for (size_t j = i + 1; j < limit; ++j)
              if (plan[seq[j]].edge_x == key.first && plan[seq[j]].edge_y == key.second) {
                limit = j;  // that test would have been skipped: later draws belong elsewhere
                break;
              }
          } else {
            ++pos[key];
          }
        }
        if (i < seq.size()) {
          *rs = snaps[i - 1];
          window = std::max<size_t>(8, window / 2);
        } else {
          window = std::min<size_t>(1024, window * 2);
        }
      }
    } else if (perm || opt.mode == FKPC_MODE_PLAIN) {
      if (evaluator) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "the level evaluator serves the batched gamma methods");
      // one test at a time; permutation methods in pcalg order
      std::map<std::pair<int, int>, size_t> pos;
      for (auto& kv : by_edge) pos[kv.first] = 0;
      for (;;) {
        int best = -1;
        for (auto& kv : by_edge) {
          const size_t at = pos[kv.first];
          if (at >= kv.second.size()) continue;
          const int cand = kv.second[at];
          if (best < 0) { best = cand; continue; }
          const Task& a = plan[cand];
          const Task& b = plan[best];
          const bool less = perm ? (a.x != b.x ? a.x < b.x : (a.y != b.y ? a.y < b.y : a.S < b.S)) : cand < best;
          if (less) best = cand;
        }
        if (best < 0) break;
        std::vector<fkpc_ci_record> rec;
        fkpc_options o1 = opt;
        o1.mode = FKPC_MODE_PLAIN;
        evaluate(*engp, {to_test(plan[best])}, o1, rs.get(), &rec, &run->stats);
        pv[best] = rec[0].p_value;
        pe[best] = rec[0].p_exact;
        fl[best] = rec[0].flags;
        counted[best] = 1;
        const std::pair<int, int> key{plan[best].edge_x, plan[best].edge_y};
        pos[key] = rec[0].p_value >= opt.alpha ? by_edge[key].size() : pos[key] + 1;
      }
    } else {
      std::vector<fkpc::Test> tests;
      tests.reserve(plan.size());
      for (const Task& t : plan) tests.push_back(to_test(t));
      std::vector<fkpc_ci_record> rec;
      if (evaluator) {
        std::vector<int> xs(tests.size()), ys(tests.size()), offs(tests.size() + 1, 0), vals;
        for (size_t i = 0; i < tests.size(); ++i) {
          xs[i] = tests[i].x;
          ys[i] = tests[i].y;
          vals.insert(vals.end(), tests[i].S.begin(), tests[i].S.end());
          offs[i + 1] = static_cast<int>(vals.size());
        }
        rec.assign(tests.size(), fkpc_ci_record{});
        const int rc = evaluator(user, level, xs.data(), ys.data(), offs.data(), vals.empty() ? nullptr : vals.data(),
                                 static_cast<int>(tests.size()), rec.data());
        if (rc != 0) throw fkpc::Error(rc, "the level evaluator failed at level " + std::to_string(level));
      } else {
        evaluate(*engp, tests, opt, nullptr, &rec, &run->stats);
      }
      for (size_t i = 0; i < plan.size(); ++i) {
        pv[i] = rec[i].p_value;
        pe[i] = rec[i].p_exact;
        fl[i] = rec[i].flags;
      }
      for (auto& kv : by_edge)
        for (int i : kv.second) {
          counted[i] = 1;
          if (pv[i] >= opt.alpha) break;
        }
    }
    // canonical replay in plan order
    bool done = true;
    int count = 0;
    std::vector<std::pair<int, int>> deleted;
    for (size_t i = 0; i < plan.size(); ++i) {
      if (!counted[i]) continue;
      const Task& t = plan[i];
      ++count;
      const size_t fwd = t.edge_x + static_cast<size_t>(p) * t.edge_y;
      const size_t rev = t.edge_y + static_cast<size_t>(p) * t.edge_x;
      if (pv[i] > run->pmax[fwd]) run->pmax[fwd] = run->pmax[rev] = pv[i];
      const bool del = pv[i] >= opt.alpha;
      if (del) {
        run->sepsets[{t.edge_x, t.edge_y}] = t.S;
        run->sepsets[{t.edge_y, t.edge_x}] = t.S;
        deleted.push_back({t.edge_x, t.edge_y});
      }
      if (t.opens) done = false;
      if (opt.collect_trace) {
        fkpc_trace_row row;
        row.level = level;
        row.task_index = static_cast<int>(i);
        row.edge_x = t.edge_x;
        row.edge_y = t.edge_y;
        row.x = t.x;
        row.y = t.y;
        row.s_offset = static_cast<int>(run->trace_s.size());
        row.s_count = static_cast<int>(t.S.size());
        row.p_value = pv[i];
        row.p_exact = pe[i];
        row.deleted = del ? 1 : 0;
        row.flags = fl[i];
        run->trace_s.insert(run->trace_s.end(), t.S.begin(), t.S.end());
        run->trace.push_back(row);
      }
    }
    for (auto& e : deleted) {
      run->adj[e.first + static_cast<size_t>(p) * e.second] = 0;
      run->adj[e.second + static_cast<size_t>(p) * e.first] = 0;
    }
    run->n_edgetests.push_back(count);
    if (done) break;
  }
}

template <class T>
T* copy_out(const std::vector<T>& v) {
  T* out = static_cast<T*>(std::malloc(sizeof(T) * std::max<size_t>(1, v.size())));
  if (!out) throw std::bad_alloc();
  if (!v.empty()) std::memcpy(out, v.data(), sizeof(T) * v.size());
  return out;
}

fkpc_result* make_result(const Run& run, const fkpc_options& options, int n, int p,
                         std::chrono::steady_clock::time_point t0) {
  fkpc_result* r = static_cast<fkpc_result*>(std::calloc(1, sizeof(fkpc_result)));
  if (!r) throw std::bad_alloc();
  r->n = n;
  r->p = p;
  r->levels = static_cast<int>(run.n_edgetests.size());
  r->adjacency = copy_out(run.adj);
  r->pmax = copy_out(run.pmax);
  std::vector<int> offs(static_cast<size_t>(p) * p + 1, 0), vals;
  for (int j = 0; j < p; ++j)
    for (int i = 0; i < p; ++i) {
      const size_t cell = i + static_cast<size_t>(p) * j;
      auto it = run.sepsets.find({i, j});
      if (it != run.sepsets.end()) vals.insert(vals.end(), it->second.begin(), it->second.end());
      offs[cell + 1] = static_cast<int>(vals.size());
    }
  r->sepset_offsets = copy_out(offs);
  r->sepset_values = copy_out(vals);
  r->n_edgetests = copy_out(run.n_edgetests);
  r->trace_rows = static_cast<int>(run.trace.size());
  r->trace = options.collect_trace ? copy_out(run.trace) : nullptr;
  r->trace_s_values = options.collect_trace ? copy_out(run.trace_s) : nullptr;
  r->stats = run.stats;
  r->elapsed_sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  r->stats.total_ms = r->elapsed_sec * 1e3;
  return r;
}

void validate_skeleton_input(int p, const int* adjacency, const int* sepset_offsets, const int* sepset_values) {
  using fkpc::Error;
  if (!adjacency || !sepset_offsets) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
  const size_t pp = static_cast<size_t>(p) * p;
  for (int i = 0; i < p; ++i)
    for (int j = 0; j < p; ++j) {
      const int a = adjacency[i + static_cast<size_t>(p) * j], b = adjacency[j + static_cast<size_t>(p) * i];
      if ((a != 0 && a != 1) || a != b || (i == j && a != 0))
        throw Error(FKPC_STATUS_INVALID_ARGUMENT, "adjacency must be a symmetric 0/1 matrix with a zero diagonal");
    }
  if (sepset_offsets[0] != 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "sepset offsets must start at 0");
  for (size_t c = 0; c < pp; ++c)
    if (sepset_offsets[c + 1] < sepset_offsets[c])
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "sepset offsets must be nondecreasing");
  if (sepset_offsets[pp] > 0 && !sepset_values) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "null sepset values");
  for (int k = 0; k < sepset_offsets[pp]; ++k)
    if (sepset_values[k] < 0 || sepset_values[k] >= p)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "sepset member out of range");
}

fkpc_orientation* make_orientation(const fkpc::Orientation& o, int p, std::chrono::steady_clock::time_point t0) {
  std::vector<fkpc_orientation_test> rows;
  std::vector<int> sets;
  for (const auto& t : o.trace) {
    fkpc_orientation_test r{};
    r.reverse = t.reverse;
    r.target = t.target;
    r.other = t.other;
    r.s_offset = static_cast<int>(sets.size());
    r.s_count = static_cast<int>(t.S.size());
    sets.insert(sets.end(), t.S.begin(), t.S.end());
    r.z_offset = static_cast<int>(sets.size());
    r.z_count = static_cast<int>(t.Z.size());
    sets.insert(sets.end(), t.Z.begin(), t.Z.end());
    r.p_value = t.p_value;
    r.rejected = t.rejected ? 1 : 0;
    rows.push_back(r);
  }
  fkpc_orientation* r = static_cast<fkpc_orientation*>(std::calloc(1, sizeof(fkpc_orientation)));
  if (!r) throw std::bad_alloc();
  try {
    r->pdag = copy_out(o.pdag);
    r->trace = copy_out(rows);
    r->set_values = copy_out(sets);
  } catch (...) {
    std::free(r->pdag);
    std::free(r->trace);
    std::free(r->set_values);
    std::free(r);
    throw;
  }
  r->p = p;
  r->collider_orientations = o.collider;
  r->rule1_orientations = o.rule1;
  r->rule2_orientations = o.rule2;
  r->rule3_orientations = o.rule3;
  r->generalized_orientations = o.generalized;
  r->regrvonps_calls = o.regrvonps_calls;
  r->residual_fits = o.residual_fits;
  r->residual_cache_hits = o.residual_cache_hits;
  r->tests = static_cast<int>(rows.size());
  r->elapsed_sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

}  // namespace

extern "C" {

int fkpc_abi_version(void) { return FKPC_ABI_VERSION; }

const char* fkpc_last_error(void) { return g_last_error.c_str(); }

void fkpc_default_options(fkpc_options* o) {
  if (!o) return;
  o->alpha = 0.1;
  o->index = 1.0;
  o->num_col = 35;
  o->max_conditioning_size = -1;
  o->ci_method = FKPC_DCC_GAMMA;
  o->hsic_sig = 1.0;
  o->permutation_replicates = 100;
  o->has_seed = 0;
  o->seed = 0;
  o->mode = FKPC_MODE_BATCHED;
  o->collect_trace = 1;
  o->device = 0;
  o->strict = 1;
  o->selection = FKPC_SELECT_MAGIC;
  o->level_graph = 0;
}

int fkpc_skeleton_run(const double* data, int n, int p, const fkpc_options* options, fkpc_result** out) {
  return guarded([&]() {
    if (!data || !options || !out) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    validate_options(*options, n, p);
    if (p > 64) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "p must be at most 64");
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    auto t0 = std::chrono::steady_clock::now();
    Run run;
    skeleton(data, n, p, *options, &run);
    *out = make_result(run, *options, n, p, t0);
  });
}

int fkpc_orient_wanpdag(const double* data, int n, int p, const int* adjacency, const int* sepset_offsets,
                        const int* sepset_values, const fkpc_options* options, fkpc_orientation** out) {
  return guarded([&]() {
    using fkpc::Error;
    if (!data || !options || !out) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    validate_options(*options, n, p);
    if (options->ci_method != FKPC_DCC_GAMMA && options->ci_method != FKPC_HSIC_GAMMA)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "the orientation covers the gamma methods");
    validate_skeleton_input(p, adjacency, sepset_offsets, sepset_values);
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    auto t0 = std::chrono::steady_clock::now();
    auto& eng = engine_for(options->device);
    eng.load(data, n, p);
    *out = make_orientation(
        fkpc::orient_wanpdag(eng, *options, data, n, p, adjacency, sepset_offsets, sepset_values), p, t0);
  });
}

int fkpc_orient_wanpdag_custom(int p, const int* adjacency, const int* sepset_offsets, const int* sepset_values,
                               double alpha, fkpc_regrvonps_evaluator evaluator, void* user,
                               fkpc_orientation** out) {
  return guarded([&]() {
    using fkpc::Error;
    if (!evaluator || !out) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (p < 2) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "need p >= 2");
    if (!(std::isfinite(alpha) && alpha > 0.0 && alpha < 1.0))
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "alpha must lie in (0, 1)");
    validate_skeleton_input(p, adjacency, sepset_offsets, sepset_values);
    auto t0 = std::chrono::steady_clock::now();
    fkpc::RegrVonPs eval = [&](int v, const std::vector<int>& S, const std::vector<int>& Z, double* pv) {
      const int rc = evaluator(user, v, S.data(), static_cast<int>(S.size()), Z.data(), static_cast<int>(Z.size()), pv);
      if (rc != 0) throw Error(rc, "orientation evaluator failed with status " + std::to_string(rc));
    };
    *out = make_orientation(fkpc::orient_wanpdag(eval, alpha, p, adjacency, sepset_offsets, sepset_values), p, t0);
  });
}

void fkpc_orientation_free(fkpc_orientation* r) {
  if (!r) return;
  std::free(r->pdag);
  std::free(r->trace);
  std::free(r->set_values);
  std::free(r);
}

int fkpc_skeleton_run_custom(const double* data, int n, int p, const fkpc_options* options,
                             fkpc_level_evaluator evaluator, void* user, fkpc_result** out) {
  return guarded([&]() {
    if (!data || !options || !out || !evaluator) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    validate_options(*options, n, p);
    if (p > 64) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "p must be at most 64");
    // no engine lock: the evaluator may call back into the batch entry points
    auto t0 = std::chrono::steady_clock::now();
    Run run;
    skeleton(data, n, p, *options, &run, evaluator, user);
    *out = make_result(run, *options, n, p, t0);
  });
}

void fkpc_result_free(fkpc_result* r) {
  if (!r) return;
  std::free(r->adjacency);
  std::free(r->pmax);
  std::free(r->sepset_offsets);
  std::free(r->sepset_values);
  std::free(r->n_edgetests);
  std::free(r->trace);
  std::free(r->trace_s_values);
  std::free(r);
}

// One batch of tests on the engine's loaded data: records into out.
void level_batch_on(fkpc::Engine& eng, const int* x, const int* y, const int* s_offsets, const int* s_values,
                    int count, const fkpc_options& opt, fkpc_ci_record* out, fkpc_stage_stats* stats,
                    std::chrono::steady_clock::time_point t0) {
  std::vector<fkpc::Test> tests(count);
  for (int t = 0; t < count; ++t) {
    tests[t].x = x[t];
    tests[t].y = y[t];
    if (s_offsets[t + 1] < s_offsets[t]) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "s_offsets must be nondecreasing");
    tests[t].S.assign(s_values + s_offsets[t], s_values + s_offsets[t + 1]);
  }
  std::unique_ptr<fkpc::RStream> rs;
  if (opt.ci_method == FKPC_DCC_PERM || opt.ci_method == FKPC_HSIC_PERM) rs.reset(new fkpc::RStream(opt.seed));
  std::vector<fkpc_ci_record> rec;
  fkpc_stage_stats acc{};
  evaluate(eng, tests, opt, rs.get(), &rec, &acc);
  std::copy(rec.begin(), rec.end(), out);
  if (stats) {
    *stats = acc;
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
}

int fkpc_ci_level_batch(const double* data, int n, int p, const int* x, const int* y, const int* s_offsets,
                        const int* s_values, int count, const fkpc_options* options, fkpc_ci_record* out,
                        fkpc_stage_stats* stats) {
  return guarded([&]() {
    if (!data || !options || !out || count < 0 || (count > 0 && (!x || !y || !s_offsets)))
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    validate_options(*options, n, p);
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    auto t0 = std::chrono::steady_clock::now();
    auto& eng = engine_for(options->device);
    eng.load(data, n, p);
    level_batch_on(eng, x, y, s_offsets, s_values, count, *options, out, stats, t0);
  });
}

int fkpc_session_load(const double* data, int n, int p, int device) {
  return guarded([&]() {
    if (!data) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    std::lock_guard<std::mutex> lock(device_mutex(device));
    auto& eng = engine_for(device);
    eng.load(data, n, p);
    slot_for(device).session = eng.load_id();
  });
}

int fkpc_session_evaluate(const int* x, const int* y, const int* s_offsets, const int* s_values, int count,
                          const fkpc_options* options, fkpc_ci_record* out, fkpc_stage_stats* stats) {
  return guarded([&]() {
    if (!options || !out || count < 0 || (count > 0 && (!x || !y || !s_offsets)))
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (options->device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    auto t0 = std::chrono::steady_clock::now();
    EngineSlot& slot = slot_for(options->device);
    if (!slot.eng || slot.session == 0 || slot.eng->load_id() != slot.session)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT,
                        "no session on this device (fkpc_session_load first; another call loaded other data)");
    validate_options(*options, slot.eng->n(), slot.eng->p());
    level_batch_on(*slot.eng, x, y, s_offsets, s_values, count, *options, out, stats, t0);
  });
}

int fkpc_ci_plain_one(const double* data, int n, int p, int x, int y, const int* s_values, int s_count,
                      const fkpc_options* options, fkpc_ci_record* out) {
  return guarded([&]() {
    if (!data || !options || !out || s_count < 0 || (s_count > 0 && !s_values))
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    validate_options(*options, n, p);
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    auto& eng = engine_for(options->device);
    eng.load(data, n, p);
    fkpc_options o = *options;
    o.mode = FKPC_MODE_PLAIN;
    std::unique_ptr<fkpc::RStream> rs;
    if (o.ci_method == FKPC_DCC_PERM || o.ci_method == FKPC_HSIC_PERM) rs.reset(new fkpc::RStream(o.seed));
    std::vector<fkpc_ci_record> rec;
    fkpc_stage_stats acc{};
    evaluate(eng, {fkpc::Test{x, y, std::vector<int>(s_values, s_values + s_count)}}, o, rs.get(), &rec, &acc);
    *out = rec[0];
  });
}

int fkpc_permutation_tables(unsigned int seed, int ci_method, int n, int replicates, int count, int* out) {
  return guarded([&]() {
    using fkpc::Error;
    if (!out && count > 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (ci_method != FKPC_DCC_PERM && ci_method != FKPC_HSIC_PERM)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation tables exist for dcc.perm and hsic.perm");
    if (n < 2 || replicates < 1 || count < 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "need n >= 2, replicates >= 1");
    fkpc::RStream rs(seed);
    const size_t per = static_cast<size_t>(replicates) * n;
    for (int t = 0; t < count; ++t) {
      if (ci_method == FKPC_DCC_PERM) rs.dcc_permutations(n, replicates, out + per * t);
      else rs.hsic_permutations(n, replicates, out + per * t);
    }
  });
}

int fkpc_regress_batch(const double* data, int n, int p, const int* target, const int* s_offsets,
                       const int* s_values, int count, const fkpc_options* options, double* residuals,
                       double* log_sp, int max_penalties, int* status) {
  return guarded([&]() {
    if (!data || !target || !s_offsets || !residuals || count < 0)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    fkpc_options o;
    fkpc_default_options(&o);
    if (options) o = *options;
    if (o.selection != FKPC_SELECT_MAGIC && o.selection != FKPC_SELECT_GN_NEWTON)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "selection must be FKPC_SELECT_MAGIC or FKPC_SELECT_GN_NEWTON");
    if (count == 0) return;  // nothing to fit: no device work
    std::lock_guard<std::mutex> lock(device_mutex(o.device));
    auto& eng = engine_for(o.device);
    eng.load(data, n, p);
    std::vector<int> tg(target, target + count);
    std::vector<std::vector<int>> sets(count);
    for (int t = 0; t < count; ++t) sets[t].assign(s_values + s_offsets[t], s_values + s_offsets[t + 1]);
    eng.regress(tg, sets, residuals, log_sp, max_penalties, status, o.selection);
  });
}

int fkpc_stat_batch(const double* residuals, int n, int m, const int* left, const int* right, int count,
                    const int* permutations, const fkpc_options* options, fkpc_ci_record* out) {
  return guarded([&]() {
    if (!residuals || !left || !right || !options || !out || count < 0 || m < 1)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    validate_options(*options, n, std::max(2, m));
    if (count == 0) return;  // no pairs: no device work
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    auto& eng = engine_for(options->device);
    eng.load(residuals, n, m);
    eng.statistics(residuals, m, std::vector<int>(left, left + count), std::vector<int>(right, right + count),
                   permutations, *options, out);
  });
}

int fkpc_batch_prepare(const double* data, int n, int p, const int* x, const int* y, const int* s_offsets,
                       const int* s_values, int count, const fkpc_options* options) {
  return guarded([&]() {
    if (!data || !options || count < 1 || !x || !y || !s_offsets)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    validate_options(*options, n, p);
    if (options->ci_method == FKPC_DCC_PERM || options->ci_method == FKPC_HSIC_PERM)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "the staged form covers the gamma methods");
    std::lock_guard<std::mutex> lock(device_mutex(options->device));
    std::vector<fkpc::Test> tests(count);
    for (int t = 0; t < count; ++t) {
      tests[t].x = x[t];
      tests[t].y = y[t];
      tests[t].S.assign(s_values + s_offsets[t], s_values + s_offsets[t + 1]);
    }
    auto& eng = engine_for(options->device);
    eng.load(data, n, p);
    eng.prepare(tests, *options, nullptr);
  });
}

int fkpc_batch_execute(int device, int repeats, double* device_ms) {
  return guarded([&]() {
    if (repeats < 1) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "repeats must be positive");
    std::lock_guard<std::mutex> lock(device_mutex(device));
    const double ms = engine_for(device).execute_timed(repeats);
    if (device_ms) *device_ms = ms;
  });
}

int fkpc_batch_collect(int device, fkpc_ci_record* out, fkpc_stage_stats* stats) {
  return guarded([&]() {
    std::lock_guard<std::mutex> lock(device_mutex(device));
    engine_for(device).collect(out, stats);
  });
}

int fkpc_batch_time_stage(int device, int stage, int repeats, double* avg_ms, double* flops_per_launch) {
  return guarded([&]() {
    std::lock_guard<std::mutex> lock(device_mutex(device));
    const double ms = engine_for(device).time_stage(stage, repeats, flops_per_launch);
    if (avg_ms) *avg_ms = ms;
  });
}

int fkpc_measure_fp64_peak(int device, double* tflops) {
  return guarded([&]() {
    std::lock_guard<std::mutex> lock(device_mutex(device));
    const double t = engine_for(device).measure_fp64_peak();
    if (tflops) *tflops = t;
  });
}

int fkpc_design_export(const double* data, int n, int p, const int* s_values, int s_count, int* q, int* m,
                       double* X, double* penalties, double* initial_log_sp) {
  return guarded([&]() {
    if (!data || !q || !m || s_count < 1 || !s_values) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    std::vector<int> S(s_values, s_values + s_count);
    std::sort(S.begin(), S.end());
    auto des = fkpc::build_design(data, n, p, S, nullptr);
    *q = des->q;
    *m = des->m;
    if (X) std::copy(des->X.begin(), des->X.end(), X);
    if (penalties) {
      const size_t qq = static_cast<size_t>(des->q) * des->q;
      std::fill(penalties, penalties + qq * des->m, 0.0);
      for (int j = 0; j < des->m; ++j) {
        const int off = des->offsets[j], dim = des->dims[j];
        for (int b = 0; b < dim; ++b)
          for (int a = 0; a < dim; ++a)
            penalties[qq * j + (off + a) + static_cast<size_t>(des->q) * (off + b)] =
                des->blocks[j][a + static_cast<size_t>(dim) * b];
      }
    }
    if (initial_log_sp) std::copy(des->initial_log_sp.begin(), des->initial_log_sp.end(), initial_log_sp);
  });
}

int fkpc_tprs_export(const double* data, int n, int p, int a, int b, int device, int* n_u, int* path, int* ok,
                     double* values, double* vectors) {
  return guarded([&]() {
    if (!data || !n_u || !path || !ok || !values || !vectors)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (n <= 5 || p < 2) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "data must be n x p with n > 5, p >= 2");
    if (device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    std::lock_guard<std::mutex> lock(device_mutex(device));
    auto& eng = engine_for(device);
    eng.load(data, n, p);
    std::vector<double> vals, U;
    eng.tprs_export(a, b, n_u, path, ok, &vals, &U);
    std::copy(vals.begin(), vals.end(), values);
    std::copy(U.begin(), U.end(), vectors);
  });
}

int fkpc_gcv_adjoint(const double* data, int n, int p, int target, const int* s_values, int s_count, int count,
                     const double* log_lambda, double* score, double* grad, double* gn_hessian,
                     double* exact_hessian, int device) {
  return guarded([&]() {
    if (!data || !s_values || (count > 0 && !log_lambda) || count < 0 || s_count < 0)
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (n <= 5 || p < 2) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "data must be n x p with n > 5, p >= 2");
    if (device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    std::lock_guard<std::mutex> lock(device_mutex(device));
    auto& eng = engine_for(device);
    eng.load(data, n, p);
    eng.adjoint(target, std::vector<int>(s_values, s_values + s_count), count, log_lambda, score, grad, gn_hessian,
                exact_hessian);
  });
}

int fkpc_get_tuning(int device, fkpc_tuning* tuning) {
  return guarded([&]() {
    if (!tuning) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    std::lock_guard<std::mutex> lock(device_mutex(device));
    *tuning = engine_for(device).tuning();
  });
}

int fkpc_set_tuning(int device, const fkpc_tuning* tuning) {
  return guarded([&]() {
    if (!tuning) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    std::lock_guard<std::mutex> lock(device_mutex(device));
    engine_for(device).set_tuning(*tuning);
  });
}

int fkpc_gamma_q_eval(int device, const double* a, const double* x, int count, double* q, int* ok) {
  return guarded([&]() {
    if (count < 0 || (count > 0 && (!a || !x || !q || !ok)))
      throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "null argument");
    if (device < 0) throw fkpc::Error(FKPC_STATUS_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    if (count == 0) return;
    fkpc::cuda_check(cudaSetDevice(device), "cudaSetDevice");
    fkpc::DevBuf<double> da, dx, dq;
    fkpc::DevBuf<int> dok;
    const size_t bytes = sizeof(double) * static_cast<size_t>(count);
    fkpc::cuda_check(cudaMemcpy(da.ensure(count), a, bytes, cudaMemcpyHostToDevice), "upload a");
    fkpc::cuda_check(cudaMemcpy(dx.ensure(count), x, bytes, cudaMemcpyHostToDevice), "upload x");
    fkpc::cuda_check(fkpc::launch_gamma_q_eval(da.get(), dx.get(), count, dq.ensure(count), dok.ensure(count), nullptr),
                     "gamma tail kernel");
    fkpc::cuda_check(cudaMemcpy(q, dq.get(), bytes, cudaMemcpyDeviceToHost), "download q");
    fkpc::cuda_check(cudaMemcpy(ok, dok.get(), sizeof(int) * static_cast<size_t>(count), cudaMemcpyDeviceToHost),
                     "download status");
  });
}

}  // extern "C"
