// C ABI (include/stopeps_gpu.h) over the engine: opaque handles, integer
// state / cache ids, status codes and the last error message.
#include "stopeps_gpu.h"
#include "pipeline.h"
#include <thread>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <memory>
#include <unordered_map>

using namespace sps;

struct sps_handle {
  std::unique_ptr<Engine> E;
  // batch workers: one engine (stream, pool, staging) per concurrent sample
  std::vector<std::unique_ptr<Engine>> workers;
  int concurrency = 1;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  sps_config cfg;
  std::vector<double> site_fields;   // per-site transverse fields; empty: cfg.h everywhere
  int var_max_sweep = 4;              // the row variational method's sweep options
  double var_threshold_sweep = 1e-8;
  std::unordered_map<int, State> states;
  std::unordered_map<int, SamplingCache> caches;
  std::unordered_map<int, int> cache_state;   // cache -> pinned state copy id
  int next_id = 1;
  std::string err;
};

namespace {

template <class F>
int guarded(sps_handle* h, F&& f) {
  if (!h) return SPS_ERR_STATE;
  try {
    f();
    h->err.clear();
    return SPS_OK;
  } catch (const Error& e) {
    h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->err = e.what();
    return SPS_ERR_ARGUMENT;
  }
}

State& get_state(sps_handle* h, int id) {
  auto it = h->states.find(id);
  if (it == h->states.end()) throw Error(SPS_ERR_STATE, "unknown state id " + std::to_string(id));
  return it->second;
}

BMPS to_bmps(const sps_handle* h, const sps_boundary* b) {
  if (!b) throw Error(SPS_ERR_ARGUMENT, "missing boundary method");
  BMPS m;
  m.chi = b->chi;
  m.space[0] = b->space0 >= 0 && b->space1 >= 0 ? b->space0 : -1;
  m.space[1] = b->space0 >= 0 && b->space1 >= 0 ? b->space1 : -1;
  if (b->absorption < 0 || b->absorption > 4) throw Error(SPS_ERR_ARGUMENT, "unknown boundary absorption");
  m.zipup = b->absorption == 1;
  m.diagonal = b->absorption == 2 || b->absorption == 4;
  m.variational = b->absorption == 3 || b->absorption == 4;
  m.max_sweep = h->var_max_sweep;
  m.threshold_sweep = h->var_threshold_sweep;
  return m;
}

Model model_of(const sps_handle* h) {
  Model m;
  m.J = h->cfg.J;
  m.h = h->cfg.h;
  m.fields = h->site_fields;
  return m;
}

FUOptions fu_of(const sps_handle* h) {
  FUOptions o;
  o.max_iterations = h->cfg.fu_max_iterations;
  o.error_tolerance = h->cfg.fu_error_tolerance;
  o.diagonal_shift = h->cfg.fu_diagonal_shift;
  o.linear_max_iterations = h->cfg.fu_linear_max_iterations;
  o.linear_tolerance = h->cfg.fu_linear_tolerance;
  return o;
}

int leg_sector(const Par& p, int c) { return par_count(p, c); }

void fill_report(const StepReport& r, sps_step_report& o) {
  o.beta = r.beta;
  o.max_state_truncation = r.max_state_truncation;
  o.max_environment_truncation = r.max_environment_truncation;
  o.max_boundary_entropy = r.max_boundary_entropy;
  o.max_solver_residual = r.max_solver_residual;
  o.max_iteration_limit_error = r.max_iteration_limit_error;
  o.bond_updates = r.bond_updates;
  o.iteration_limit_hits = r.iteration_limit_hits;
  o.stop_error_tolerance = r.stop_reasons[0];
  o.stop_iteration_limit = r.stop_reasons[1];
  o.stop_residual_fallback = r.stop_reasons[2];
  o.stop_disabled = r.stop_reasons[3];
  o.linear_unconverged_updates = r.linear_unconverged;
  o.repairs = r.repairs;
  o.fallbacks = r.fallbacks;
  double sum = 0;
  for (double v : r.log_normalizations) sum += v;
  o.log_normalization_sum = sum;
}

void fill_energy(const EnergyResult& r, sps_energy& o) {
  o.energy_total = r.energy_total;
  o.energy_per_site = r.energy_per_site;
  o.log_norm = r.log_norm;
  o.tensor_log_norm = r.tensor_log_norm;
  o.max_environment_truncation = r.max_env_trunc;
  o.x_sum = r.x_sum;
  o.zz_sum = r.zz_sum;
}

// Run fn(engine, i) for i in [0, n): serially on the handle's engine when the
// concurrency is 1, else on min(concurrency, n) worker engines (own CUDA
// stream, memory pool and staging ring each), worker w taking i = w, w + W,
// ...  The workers' streams wait for the handle's stream at the start and the
// handle's stream waits for them at the end, so events recorded on the
// handle's stream bracket the whole batch and every buffer that changes
// hands between engines is used in stream order.  The first error (lowest
// worker) is rethrown after all workers have finished.
template <class F>
void run_batch(sps_handle* h, int n, F&& fn) {
  if (n < 0) throw Error(SPS_ERR_ARGUMENT, "negative batch size");
  const int W = std::min<int>(h->concurrency, std::max(n, 1));
  Engine& M = *h->E;
  if (W <= 1) {
    for (int i = 0; i < n; ++i) fn(M, i);
    return;
  }
  while ((int)h->workers.size() < W) {
    h->workers.push_back(std::make_unique<Engine>(M.device));
    h->workers.back()->ctas_cap = M.num_sms / h->concurrency;
    h->workers.back()->force_repair = M.force_repair;
    h->workers.back()->full_spectrum = M.full_spectrum;
    h->workers.back()->sweep_cap = M.sweep_cap;
    h->workers.back()->eigh_multi_min = M.eigh_multi_min;
    h->workers.back()->precision = M.precision;
    h->workers.back()->autotune = M.autotune;
    h->workers.back()->profile = M.profile;
  }
  cudaEvent_t start;
  SPS_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  SPS_CUDA(cudaEventRecord(start, M.stream));
  for (int w = 0; w < W; ++w) SPS_CUDA(cudaStreamWaitEvent(h->workers[w]->stream, start, 0));
  std::vector<int> codes(W, SPS_OK);
  std::vector<std::string> msgs(W);
  std::vector<std::thread> threads;
  for (int w = 0; w < W; ++w)
    threads.emplace_back([&, w] {
      try {
        SPS_CUDA(cudaSetDevice(M.device));
        Engine& E = *h->workers[w];
        for (int i = w; i < n; i += W) fn(E, i);
      } catch (const Error& e) {
        codes[w] = e.code;
        msgs[w] = e.what();
      } catch (const std::exception& e) {
        codes[w] = SPS_ERR_ARGUMENT;
        msgs[w] = e.what();
      }
    });
  for (auto& t : threads) t.join();
  for (int w = 0; w < W; ++w) {
    cudaEvent_t done;
    SPS_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    SPS_CUDA(cudaEventRecord(done, h->workers[w]->stream));
    SPS_CUDA(cudaStreamWaitEvent(M.stream, done, 0));
    SPS_CUDA(cudaEventDestroy(done));
  }
  SPS_CUDA(cudaEventDestroy(start));
  for (int w = 0; w < W; ++w)
    if (codes[w] != SPS_OK) throw Error(codes[w], msgs[w]);
}

// distinct states of a batch call (a state updated in place appears once)
std::vector<State*> batch_states(sps_handle* h, int n, const int32_t* ids) {
  if (n > 0 && !ids) throw Error(SPS_ERR_ARGUMENT, "missing state ids");
  std::vector<State*> out(n);
  for (int i = 0; i < n; ++i) {
    out[i] = &get_state(h, ids[i]);
    for (int j = 0; j < i; ++j)
      if (ids[j] == ids[i]) throw Error(SPS_ERR_ARGUMENT, "a state id appears twice in one batch");
  }
  return out;
}

bool sorted_leg(const Par& p) {
  for (size_t i = 1; i < p->size(); ++i)
    if ((*p)[i] < (*p)[i - 1]) return false;
  return true;
}

}  // namespace

extern "C" {

int sps_create(const sps_config* cfg, sps_handle** out) {
  if (!cfg || !out) return SPS_ERR_ARGUMENT;
  *out = nullptr;
  auto h = new sps_handle();
  h->cfg = *cfg;
  if (cfg->Lx < 1 || cfg->Ly < 1 || (cfg->trotter_order != 1 && cfg->trotter_order != 2) ||
      cfg->fu_max_iterations < 0 || cfg->fu_linear_max_iterations < 1) {
    delete h;
    return SPS_ERR_ARGUMENT;
  }
  try {
    h->E.reset(new Engine(cfg->device));
  } catch (const Error& e) {
    delete h;
    return e.code;
  }
  *out = h;
  return SPS_OK;
}

void sps_destroy(sps_handle* h) {
  if (!h) return;
  if (h->t0) cudaEventDestroy(h->t0);
  if (h->t1) cudaEventDestroy(h->t1);
  h->caches.clear();
  h->states.clear();
  delete h;
}

int sps_last_error(const sps_handle* h, char* buf, size_t n) {
  if (!h || !buf || n == 0) return SPS_ERR_ARGUMENT;
  std::strncpy(buf, h->err.c_str(), n - 1);
  buf[n - 1] = 0;
  return SPS_OK;
}

int sps_counters(sps_handle* h, long long* launches, double* flops) {
  return guarded(h, [&] {
    long long n = h->E->launches;
    double f = h->E->flops;
    for (auto& w : h->workers) {
      n += w->launches;
      f += w->flops;
    }
    if (launches) *launches = n;
    if (flops) *flops = f;
  });
}

int sps_set_concurrency(sps_handle* h, int32_t samples) {
  return guarded(h, [&] {
    if (samples < 1 || samples > 16) throw Error(SPS_ERR_ARGUMENT, "concurrency must be in 1..16");
    h->concurrency = samples;
    for (auto& w : h->workers) w->ctas_cap = h->E->num_sms / samples;
  });
}

int sps_set_sm_share(sps_handle* h, int32_t ctas) {
  return guarded(h, [&] {
    if (ctas < 0 || ctas > h->E->num_sms) throw Error(SPS_ERR_ARGUMENT, "sps_set_sm_share: ctas must be in 0..SMs");
    h->E->ctas_cap = ctas;
  });
}

int sps_set_precision(sps_handle* h, int32_t mode) {
  return guarded(h, [&] {
    if (mode < 0 || mode > 3) throw Error(SPS_ERR_ARGUMENT, "sps_set_precision: mode must be 0..3");
    h->E->precision = mode;
    for (auto& w : h->workers) w->precision = mode;
  });
}

int sps_set_autotune(sps_handle* h, int32_t enable) {
  return guarded(h, [&] {
    h->E->autotune = enable != 0;
    for (auto& w : h->workers) w->autotune = enable != 0;
  });
}

int sps_autotune_report(sps_handle* h, char* buf, size_t n) {
  return guarded(h, [&] {
    const std::string js = tune::report_json();
    if (!buf || js.size() + 1 > n) throw Error(SPS_ERR_ARGUMENT, "buffer too small");
    std::memcpy(buf, js.c_str(), js.size() + 1);
  });
}

int sps_set_truncated_svd(sps_handle* h, int32_t method) {
  return guarded(h, [&] {
    if (method != 0 && method != 1) throw Error(SPS_ERR_ARGUMENT, "sps_set_truncated_svd: method is 0 or 1");
    h->E->full_spectrum = method == 1;
    for (auto& w : h->workers) w->full_spectrum = method == 1;
  });
}

int sps_set_variational(sps_handle* h, int32_t max_sweep, double threshold_sweep) {
  return guarded(h, [&] {
    if (max_sweep < 1) throw Error(SPS_ERR_ARGUMENT, "max_sweep must be positive");
    if (!(std::isfinite(threshold_sweep) && threshold_sweep >= 0))
      throw Error(SPS_ERR_ARGUMENT, "threshold_sweep must be finite and nonnegative");
    h->var_max_sweep = max_sweep;
    h->var_threshold_sweep = threshold_sweep;
  });
}

int sps_lognorm_variational(sps_handle* h, int32_t state_id, const sps_boundary* method, sps_lognorm_result* out,
                            int32_t* counts, double* max_relative_change) {
  return guarded(h, [&] {
    LogNorm r = lognorm(*h->E, get_state(h, state_id), to_bmps(h, method));
    if (out) {
      out->log_norm = r.log_norm;
      out->tensor_log_norm = r.tensor_log_norm;
      out->max_environment_truncation = r.max_env_trunc;
    }
    // _variational_summary (diagonal_variational.jl:40-46)
    int layers = (int)r.variational.size(), max_sweeps = 0, limit = 0, fallbacks = 0;
    double change = 0;
    for (const auto& v : r.variational) {
      max_sweeps = std::max(max_sweeps, v.sweeps);
      limit += v.stop_reason == VariationalRecord::SWEEP_LIMIT;
      fallbacks += v.fallback;
      if (std::isfinite(v.relative_change)) change = std::max(change, v.relative_change);
    }
    if (counts) {
      counts[0] = layers;
      counts[1] = max_sweeps;
      counts[2] = limit;
      counts[3] = fallbacks;
    }
    if (max_relative_change) *max_relative_change = change;
  });
}

int sps_lognorm_gradient(sps_handle* h, int32_t state_id, const sps_boundary* method, int32_t checkpoint_rows,
                         double* log_norm, double* grads, int64_t capacity) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    LognormGradient r = lognorm_gradient(*h->E, s, to_bmps(h, method), checkpoint_rows != 0);
    if (log_norm) *log_norm = r.log_norm;
    if (grads) {
      int64_t off = 0;
      for (auto& t : r.grads) {
        if (off + t.size() > capacity) throw Error(SPS_ERR_ARGUMENT, "buffer too small");
        auto v = h->E->download(t);
        std::memcpy(grads + off, v.data(), v.size() * sizeof(double));
        off += t.size();
      }
    }
  });
}

int sps_lognorm_field_gradient(sps_handle* h, int32_t state_id, const sps_boundary* method, int32_t checkpoint_rows,
                               double* log_norm, double* site_x, double* d_fields) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    FieldGradient r = lognorm_field_gradient(*h->E, s, to_bmps(h, method), checkpoint_rows != 0);
    if (log_norm) *log_norm = r.log_norm;
    if (site_x) std::copy(r.site_x.begin(), r.site_x.end(), site_x);
    if (d_fields) std::copy(r.d_fields.begin(), r.d_fields.end(), d_fields);
  });
}

int sps_set_site_fields(sps_handle* h, int32_t n, const double* fields) {
  return guarded(h, [&] {
    if (n == 0) {
      h->site_fields.clear();
      return;
    }
    if (n != h->cfg.Lx * h->cfg.Ly || !fields)
      throw Error(SPS_ERR_ARGUMENT, "sps_set_site_fields: n must be Lx*Ly (or 0 to clear)");
    std::vector<double> f(fields, fields + n);
    for (double v : f)
      if (!std::isfinite(v)) throw Error(SPS_ERR_ARGUMENT, "sps_set_site_fields: nonfinite field");
    h->site_fields = std::move(f);
  });
}

int sps_set_injection(sps_handle* h, int32_t force_repair, int32_t svd_sweep_cap, int32_t multi_cta_eigh_min) {
  return guarded(h, [&] {
    if (svd_sweep_cap < 0 || multi_cta_eigh_min < 0) throw Error(SPS_ERR_ARGUMENT, "sps_set_injection: negative value");
    const int em = multi_cta_eigh_min > 0 ? multi_cta_eigh_min : 1024;
    h->E->force_repair = force_repair != 0;
    h->E->sweep_cap = svd_sweep_cap;
    h->E->eigh_multi_min = em;
    for (auto& w : h->workers) {
      w->force_repair = force_repair != 0;
      w->sweep_cap = svd_sweep_cap;
      w->eigh_multi_min = em;
    }
  });
}

int sps_set_profile(sps_handle* h, int32_t enable) {
  return guarded(h, [&] {
    const int level = enable < 0 ? 0 : (enable > 2 ? 2 : enable);
    h->E->reset_stats();
    h->E->profile = level;
    for (auto& w : h->workers) {
      w->reset_stats();
      w->profile = level;
    }
  });
}

int sps_kernel_stats_json(sps_handle* h, char* buf, size_t n) {
  return guarded(h, [&] {
    // the handle's engine and every batch worker (per-kernel times add up
    // over the engines; under concurrency each is the kernel's own duration
    // on its stream while the others run beside it)
    auto st = h->E->kernel_stats();
    for (auto& w : h->workers)
      for (auto& kv : w->kernel_stats()) {
        auto& k = st[kv.first];
        k.ms += kv.second.ms;
        k.flops += kv.second.flops;
        k.bytes += kv.second.bytes;
        k.count += kv.second.count;
      }
    std::string js = "{";
    bool first = true;
    char tmp[512];
    for (auto& kv : st) {
      std::snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"ms\": %.6f, \"count\": %lld, \"flops\": %.6e, \"bytes\": %.6e}",
                    first ? "" : ", ", kv.first.c_str(), kv.second.ms, kv.second.count, kv.second.flops,
                    kv.second.bytes);
      js += tmp;
      first = false;
    }
    js += "}";
    if (!buf || js.size() + 1 > n) throw Error(SPS_ERR_ARGUMENT, "buffer too small");
    std::memcpy(buf, js.c_str(), js.size() + 1);
  });
}

int sps_timer_start(sps_handle* h) {
  return guarded(h, [&] {
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaEventRecord(h->t0, h->E->stream));
  });
}

int sps_timer_stop(sps_handle* h, double* ms) {
  return guarded(h, [&] {
    SPS_CUDA(cudaEventRecord(h->t1, h->E->stream));
    SPS_CUDA(cudaEventSynchronize(h->t1));
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    if (ms) *ms = f;
  });
}

static double* dev_copy(Engine& E, Buf& b, const double* h, size_t n) {
  b = E.alloc(sizeof(double) * std::max<size_t>(n, 1));
  SPS_CUDA(cudaMemcpyAsync(b->ptr, h, sizeof(double) * n, cudaMemcpyHostToDevice, E.stream));
  return (double*)b->ptr;
}

int sps_la_svd(sps_handle* h, int32_t m, int32_t n, const double* a, double* u, double* s, double* vt,
               int32_t* sweeps, double* ms) {
  return guarded(h, [&] {
    Engine& E = *h->E;
    if (m < 1 || n < 1) throw Error(SPS_ERR_ARGUMENT, "empty matrix");
    bool tall = m >= n;
    int mm = tall ? m : n, nn = tall ? n : m;
    std::vector<double> at;
    const double* src = a;
    if (!tall) {   // work on a^T
      at.resize((size_t)m * n);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) at[j + (size_t)i * n] = a[i + (size_t)j * m];
      src = at.data();
    }
    Buf ba, bq, br, bs;
    double* da = dev_copy(E, ba, src, (size_t)mm * nn);
    bq = E.alloc(sizeof(double) * (size_t)mm * nn);
    br = E.alloc(sizeof(double) * (size_t)nn * nn);
    bs = E.alloc(sizeof(double) * nn);
    la::MatDesc d{da, (double*)bq->ptr, (double*)br->ptr, (double*)bs->ptr, mm, nn, mm, mm, nn};
    SPS_CUDA(cudaMemsetAsync(E.dflag + 1, 0, sizeof(int), E.stream));
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaEventRecord(h->t0, E.stream));
    if (la::svd_is_big(mm, nn)) la::svd_big(E, {d});
    else la::svd_batched(E, {d});
    SPS_CUDA(cudaEventRecord(h->t1, E.stream));
    std::vector<double> U((size_t)mm * nn), V((size_t)nn * nn), S(nn);
    SPS_CUDA(cudaMemcpyAsync(U.data(), d.q, U.size() * 8, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(V.data(), d.r, V.size() * 8, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(S.data(), d.s, S.size() * 8, cudaMemcpyDeviceToHost, E.stream));
    int sw = 0;
    SPS_CUDA(cudaMemcpyAsync(&sw, E.dflag + 1, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    E.check_flag("sps_la_svd");
    if (ms) *ms = f;
    if (sweeps) *sweeps = sw;
    int k = nn;
    if (s) std::copy(S.begin(), S.end(), s);
    // a = U S V^T (tall) ; a^T = U S V^T -> a = V S U^T (wide)
    for (int l = 0; l < k; ++l) {
      for (int i = 0; i < m; ++i)
        if (u) u[i + (size_t)l * m] = tall ? U[i + (size_t)l * mm] : V[i + (size_t)l * nn];
      for (int j = 0; j < n; ++j)
        if (vt) vt[l + (size_t)j * k] = tall ? V[j + (size_t)l * nn] : U[j + (size_t)l * mm];
    }
  });
}

int sps_la_svd_left(sps_handle* h, int32_t m, int32_t n, const double* a, double* u, double* s, int32_t* sweeps,
                    double* ms) {
  return guarded(h, [&] {
    Engine& E = *h->E;
    if (m < n || n < 1) throw Error(SPS_ERR_ARGUMENT, "sps_la_svd_left needs m >= n >= 1");
    Buf ba, bq, bs;
    double* da = dev_copy(E, ba, a, (size_t)m * n);
    bq = E.alloc(sizeof(double) * (size_t)m * n);
    bs = E.alloc(sizeof(double) * n);
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaMemsetAsync(E.dflag + 1, 0, sizeof(int), E.stream));
    SPS_CUDA(cudaEventRecord(h->t0, E.stream));
    la::jacobi_left(E, {la::MatDesc{da, (double*)bq->ptr, nullptr, (double*)bs->ptr, m, n, m, m, 0}});
    SPS_CUDA(cudaEventRecord(h->t1, E.stream));
    SPS_CUDA(cudaMemcpyAsync(u, bq->ptr, sizeof(double) * (size_t)m * n, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(s, bs->ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, E.stream));
    int sw = 0;
    SPS_CUDA(cudaMemcpyAsync(&sw, E.dflag + 1, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    E.check_flag("sps_la_svd_left");
    if (ms) *ms = f;
    if (sweeps) *sweeps = sw;
  });
}

int sps_la_svd_topk(sps_handle* h, int32_t m, int32_t n, int32_t k, const double* a, int32_t gram, double rtol,
                    double* u, double* s, double* v, int32_t* iterations, double* ms) {
  return guarded(h, [&] {
    Engine& E = *h->E;
    if (k < 1 || la::topk_block_size(k, m, n) == 0)
      throw Error(SPS_ERR_ARGUMENT, "sps_la_svd_topk needs 1 <= k and a block at least twice the iteration width");
    if (!la::topk_fits(k, m, n, 1, E)) throw Error(SPS_ERR_ARGUMENT, "sps_la_svd_topk: block too large");
    Buf ba, bu;
    double* da = dev_copy(E, ba, a, (size_t)m * n);
    bu = E.alloc(sizeof(double) * (size_t)(m + n) * k);
    std::vector<la::TopkDesc> ds(1);
    ds[0].M = da;
    ds[0].m = m;
    ds[0].n = n;
    ds[0].k = k;
    ds[0].U = (double*)bu->ptr;
    ds[0].V = ds[0].U + (size_t)m * k;
    ds[0].gram = gram != 0;
    if (!(rtol >= 0.0)) throw Error(SPS_ERR_ARGUMENT, "sps_la_svd_topk: rtol must be >= 0");
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaEventRecord(h->t0, E.stream));
    la::svd_topk(E, ds, rtol > 0.0 ? rtol : 5e-14);
    if (ds[0].status == 4 && ds[0].gram) {   // wanted directions lost on M M^T: again on M, as the engine does
      ds[0].gram = false;
      la::svd_topk(E, ds, rtol > 0.0 ? rtol : 5e-14);
    }
    SPS_CUDA(cudaEventRecord(h->t1, E.stream));
    SPS_CUDA(cudaMemcpyAsync(u, ds[0].U, sizeof(double) * (size_t)m * k, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(v, ds[0].V, sizeof(double) * (size_t)n * k, cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    for (int i = 0; i < k; ++i) s[i] = ds[0].s[i];
    if (ms) *ms = f;
    if (iterations) *iterations = ds[0].iterations;
    if (ds[0].status != 0)
      throw Error(SPS_ERR_CONVERGENCE, "sps_la_svd_topk: subspace iteration did not converge (status " +
                                           std::to_string(ds[0].status) + ")");
  });
}

int sps_la_gemm(sps_handle* h, int32_t transpose_a, int32_t m, int32_t n, int32_t k, double alpha, const double* a,
                const double* b, double beta, double* c, double* ms) {
  return guarded(h, [&] {
    Engine& E = *h->E;
    if (m < 1 || n < 1 || k < 0) throw Error(SPS_ERR_ARGUMENT, "sps_la_gemm: bad sizes");
    Buf ba, bb, bc;
    double* da = dev_copy(E, ba, a, (size_t)m * k);
    double* db = dev_copy(E, bb, b, (size_t)k * n);
    double* dc = dev_copy(E, bc, c, (size_t)m * n);
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaEventRecord(h->t0, E.stream));
    la::dgemm_cm(E, transpose_a != 0, m, n, k, alpha, da, transpose_a ? std::max(k, 1) : m, db, std::max(k, 1), beta,
                 dc, m);
    SPS_CUDA(cudaEventRecord(h->t1, E.stream));
    SPS_CUDA(cudaMemcpyAsync(c, dc, sizeof(double) * (size_t)m * n, cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    if (ms) *ms = f;
  });
}

int sps_la_gemm_mixed(sps_handle* h, int32_t mode, int32_t m, int32_t n, int32_t k, const double* a,
                      const double* b, double* c, double* ms) {
  return guarded(h, [&] {
    Engine& E = *h->E;
    if (m < 1 || n < 1 || k < 1) throw Error(SPS_ERR_ARGUMENT, "sps_la_gemm_mixed: bad sizes");
    if (mode < 1 || mode > 3) throw Error(SPS_ERR_ARGUMENT, "sps_la_gemm_mixed: mode must be 1..3");
    Buf ba, bb, bc, t[6];
    double* da = dev_copy(E, ba, a, (size_t)m * k);
    double* db = dev_copy(E, bb, b, (size_t)k * n);
    bc = E.alloc(sizeof(double) * (size_t)m * n);
    double* dc = (double*)bc->ptr;
    // row-major a (m x k), b (k x n), c (m x n) as offset tables
    std::vector<int64_t> ra(m), ca(k), rb(k), cb(n), rc(m), cc(n);
    for (int i = 0; i < m; ++i) ra[i] = (int64_t)i * k, rc[i] = (int64_t)i * n;
    for (int i = 0; i < k; ++i) ca[i] = i, rb[i] = (int64_t)i * n;
    for (int i = 0; i < n; ++i) cb[i] = i, cc[i] = i;
    const int64_t* dra = E.upload_i64(ra, t[0]);
    const int64_t* dca = E.upload_i64(ca, t[1]);
    const int64_t* drb = E.upload_i64(rb, t[2]);
    const int64_t* dcb = E.upload_i64(cb, t[3]);
    const int64_t* drc = E.upload_i64(rc, t[4]);
    const int64_t* dcc = E.upload_i64(cc, t[5]);
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaEventRecord(h->t0, E.stream));
    tc::gemm_block(E, mode, da, dra, dca, 1, db, drb, dcb, 1, dc, drc, dcc, m, n, k, 1.0);
    SPS_CUDA(cudaEventRecord(h->t1, E.stream));
    SPS_CUDA(cudaMemcpyAsync(c, dc, sizeof(double) * (size_t)m * n, cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    E.check_flag("sps_la_gemm_mixed");
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    if (ms) *ms = f;
  });
}

int sps_la_qr(sps_handle* h, int32_t m, int32_t n, const double* a, double* q, double* r, double* ms) {
  return guarded(h, [&] {
    Engine& E = *h->E;
    if (m < 1 || n < 1) throw Error(SPS_ERR_ARGUMENT, "empty matrix");
    int k = std::min(m, n);
    Buf ba, bq, br, bs;
    double* da = dev_copy(E, ba, a, (size_t)m * n);
    bq = E.alloc(sizeof(double) * (size_t)m * k);
    br = E.alloc(sizeof(double) * (size_t)k * n);
    bs = E.alloc(sizeof(double) * k);
    if (!h->t0) {
      SPS_CUDA(cudaEventCreate(&h->t0));
      SPS_CUDA(cudaEventCreate(&h->t1));
    }
    SPS_CUDA(cudaEventRecord(h->t0, E.stream));
    if (la::qr_is_big(m, n)) la::qr_big(E, da, m, n, m, (double*)bq->ptr, m, (double*)br->ptr, k);
    else la::qr_batched(E, {la::MatDesc{da, (double*)bq->ptr, (double*)br->ptr, (double*)bs->ptr, m, n, m, m, k}});
    SPS_CUDA(cudaEventRecord(h->t1, E.stream));
    SPS_CUDA(cudaMemcpyAsync(q, bq->ptr, sizeof(double) * (size_t)m * k, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(r, br->ptr, sizeof(double) * (size_t)k * n, cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    float f = 0;
    SPS_CUDA(cudaEventElapsedTime(&f, h->t0, h->t1));
    E.check_flag("sps_la_qr");
    if (ms) *ms = f;
  });
}

int sps_identity_pepo(sps_handle* h, int32_t* state_id) {
  return guarded(h, [&] {
    int id = h->next_id++;
    h->states[id] = identity_pepo(*h->E, h->cfg.Lx, h->cfg.Ly);
    *state_id = id;
  });
}

int sps_state_upload(sps_handle* h, int32_t is_pepo, double beta, double log_amplitude, const int32_t* leg_dims,
                     const double* data, int32_t* state_id) {
  return guarded(h, [&] {
    if (!leg_dims || !data || !state_id) throw Error(SPS_ERR_ARGUMENT, "null pointer");
    State s;
    s.Lx = h->cfg.Lx;
    s.Ly = h->cfg.Ly;
    s.beta = beta;
    s.log_amplitude = log_amplitude;
    s.pepo = is_pepo != 0;
    const double* ptr = data;
    for (int i = 0; i < s.Lx * s.Ly; ++i) {
      std::vector<Par> legs;
      for (int k = 0; k < 6; ++k) {
        int n0 = leg_dims[(i * 6 + k) * 2], n1 = leg_dims[(i * 6 + k) * 2 + 1];
        if (n0 < 0 || n1 < 0 || n0 + n1 == 0) throw Error(SPS_ERR_ARGUMENT, "invalid leg dimensions");
        legs.push_back(make_par(n0, n1));
      }
      Tensor t = h->E->upload(legs, ptr);
      ptr += t.size();
      s.sites.push_back(t);
    }
    int id = h->next_id++;
    h->states[id] = std::move(s);
    *state_id = id;
  });
}

int sps_state_layout(sps_handle* h, int32_t state_id, int32_t* leg_dims, int64_t* total) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    int64_t tot = 0;
    for (int i = 0; i < s.Lx * s.Ly; ++i) {
      const Tensor& t = s.sites[i];
      for (int k = 0; k < 6; ++k) {
        if (!sorted_leg(t.legs[k])) throw Error(SPS_ERR_STATE, "site leg is not sector sorted");
        if (leg_dims) {
          leg_dims[(i * 6 + k) * 2] = leg_sector(t.legs[k], 0);
          leg_dims[(i * 6 + k) * 2 + 1] = leg_sector(t.legs[k], 1);
        }
      }
      tot += t.size();
    }
    if (total) *total = tot;
  });
}

int sps_state_download(sps_handle* h, int32_t state_id, double* data, int64_t capacity) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    int64_t off = 0;
    for (auto& t : s.sites) {
      if (off + t.size() > capacity) throw Error(SPS_ERR_ARGUMENT, "buffer too small");
      auto v = h->E->download(t);
      std::memcpy(data + off, v.data(), v.size() * sizeof(double));
      off += t.size();
    }
  });
}

int sps_state_info(sps_handle* h, int32_t state_id, double* beta, double* log_amplitude, int32_t* is_pepo) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    if (beta) *beta = s.beta;
    if (log_amplitude) *log_amplitude = s.log_amplitude;
    if (is_pepo) *is_pepo = s.pepo ? 1 : 0;
  });
}

int sps_state_set_beta(sps_handle* h, int32_t state_id, double beta) {
  return guarded(h, [&] { get_state(h, state_id).beta = beta; });
}

int sps_state_copy(sps_handle* h, int32_t state_id, int32_t* new_id) {
  return guarded(h, [&] {
    State c = get_state(h, state_id);
    for (auto& t : c.sites) t = clone(*h->E, t);
    int id = h->next_id++;
    h->states[id] = std::move(c);
    *new_id = id;
  });
}

int sps_state_free(sps_handle* h, int32_t state_id) {
  return guarded(h, [&] {
    if (!h->states.erase(state_id)) throw Error(SPS_ERR_STATE, "unknown state id");
  });
}

int sps_normalize_state(sps_handle* h, int32_t state_id, double* log_normalizations) {
  return guarded(h, [&] {
    auto v = normalize_state(*h->E, get_state(h, state_id));
    if (log_normalizations) std::memcpy(log_normalizations, v.data(), v.size() * sizeof(double));
  });
}

int sps_evolution_step(sps_handle* h, int32_t state_id, double delta, int32_t D, const int32_t* space,
                       const sps_boundary* environment, sps_step_report* report) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    int sp[2] = {-1, -1};
    if (space) {
      sp[0] = space[0];
      sp[1] = space[1];
    }
    StepReport r = evolution_step(*h->E, s, model_of(h), delta, D, fu_of(h), to_bmps(h, environment),
                                  h->cfg.trotter_order, sp, h->cfg.record_boundary_entropy != 0);
    if (report) fill_report(r, *report);
  });
}

int sps_evolution_step_batch(sps_handle* h, int32_t n, const int32_t* state_ids, const double* deltas, int32_t D,
                             const int32_t* space, const sps_boundary* environment, sps_step_report* reports) {
  return guarded(h, [&] {
    if (n > 0 && !deltas) throw Error(SPS_ERR_ARGUMENT, "missing deltas");
    std::vector<State*> st = batch_states(h, n, state_ids);
    int sp[2] = {-1, -1};
    if (space) {
      sp[0] = space[0];
      sp[1] = space[1];
    }
    const BMPS m = to_bmps(h, environment);
    const Model md = model_of(h);
    const FUOptions o = fu_of(h);
    run_batch(h, n, [&](Engine& E, int i) {
      StepReport r = evolution_step(E, *st[i], md, deltas[i], D, o, m, h->cfg.trotter_order, sp,
                                    h->cfg.record_boundary_entropy != 0);
      if (reports) fill_report(r, reports[i]);
    });
  });
}

int sps_lognorm(sps_handle* h, int32_t state_id, const sps_boundary* method, sps_lognorm_result* out) {
  return guarded(h, [&] {
    LogNorm r = lognorm(*h->E, get_state(h, state_id), to_bmps(h, method));
    if (out) {
      out->log_norm = r.log_norm;
      out->tensor_log_norm = r.tensor_log_norm;
      out->max_environment_truncation = r.max_env_trunc;
    }
  });
}

int sps_measure_energy(sps_handle* h, int32_t state_id, const sps_boundary* method, sps_energy* out,
                       double* site_x, double* se_north, double* se_south) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    EnergyResult r = measure_energy(*h->E, s, model_of(h), to_bmps(h, method), h->cfg.record_boundary_entropy != 0);
    if (out) fill_energy(r, *out);
    if (site_x) std::memcpy(site_x, r.site_x.data(), r.site_x.size() * sizeof(double));
    // the diagonal method's profiles are per site (northwest, southeast)
    const auto& a = r.entropy.northwest.empty() ? r.entropy.north : r.entropy.northwest;
    const auto& b = r.entropy.southeast.empty() ? r.entropy.south : r.entropy.southeast;
    if (se_north && r.entropy.profile) std::memcpy(se_north, a.data(), a.size() * sizeof(double));
    if (se_south && r.entropy.profile) std::memcpy(se_south, b.data(), b.size() * sizeof(double));
  });
}

int sps_measure_energy_batch(sps_handle* h, int32_t n, const int32_t* state_ids, const sps_boundary* method,
                             sps_energy* out, double* site_x) {
  return guarded(h, [&] {
    std::vector<State*> st = batch_states(h, n, state_ids);
    const BMPS m = to_bmps(h, method);
    const Model md = model_of(h);
    const size_t L = (size_t)h->cfg.Lx * h->cfg.Ly;
    run_batch(h, n, [&](Engine& E, int i) {
      EnergyResult r = measure_energy(E, *st[i], md, m, h->cfg.record_boundary_entropy != 0);
      if (out) fill_energy(r, out[i]);
      if (site_x) std::memcpy(site_x + i * L, r.site_x.data(), std::min(L, r.site_x.size()) * sizeof(double));
    });
  });
}

int sps_lognorm_batch(sps_handle* h, int32_t n, const int32_t* state_ids, const sps_boundary* method,
                      sps_lognorm_result* out) {
  return guarded(h, [&] {
    std::vector<State*> st = batch_states(h, n, state_ids);
    const BMPS m = to_bmps(h, method);
    run_batch(h, n, [&](Engine& E, int i) {
      LogNorm r = lognorm(E, *st[i], m);
      if (out) {
        out[i].log_norm = r.log_norm;
        out[i].tensor_log_norm = r.tensor_log_norm;
        out[i].max_environment_truncation = r.max_env_trunc;
      }
    });
  });
}

static void fill_sample(const SampleResult& r, sps_sample_report& o) {
  o.log_probability = r.log_probability;
  o.max_environment_truncation = r.max_env_trunc;
  o.near_boundary = r.near_boundary;
  o.metric_repairs = r.metric_repairs;
  o.zero_proposals = r.zero_proposals;
  o.min_relative_eigenvalue = r.min_relative_eigenvalue;
}

int sps_sampling_cache(sps_handle* h, int32_t pepo_id, const sps_boundary* method, int32_t* cache_id) {
  return guarded(h, [&] {
    State& s = get_state(h, pepo_id);
    if (!s.pepo) throw Error(SPS_ERR_ARGUMENT, "auxiliary sampling requires a PEPO");
    // the cache keeps its own reference to the PEPO tensors
    int sid = h->next_id++;
    h->states[sid] = s;
    int id = h->next_id++;
    h->caches[id] = make_sampling_cache(*h->E, h->states[sid], to_bmps(h, method));
    h->cache_state[id] = sid;
    *cache_id = id;
  });
}

int sps_sampling_cache_kind(sps_handle* h, int32_t state_id, const sps_boundary* method, int32_t kind,
                            int32_t* cache_id) {
  return guarded(h, [&] {
    State& s = get_state(h, state_id);
    if (kind == KIND_AUXILIARY && !s.pepo) throw Error(SPS_ERR_ARGUMENT, "auxiliary sampling requires a PEPO");
    if (kind == KIND_PHYSICAL && s.pepo) throw Error(SPS_ERR_ARGUMENT, "proposal requires PEPS");
    int sid = h->next_id++;
    h->states[sid] = s;
    int id = h->next_id++;
    h->caches[id] = make_sampling_cache(*h->E, h->states[sid], to_bmps(h, method), kind);
    h->cache_state[id] = sid;
    *cache_id = id;
  });
}

int sps_sampling_cache_free(sps_handle* h, int32_t cache_id) {
  return guarded(h, [&] {
    auto it = h->caches.find(cache_id);
    if (it == h->caches.end()) throw Error(SPS_ERR_STATE, "unknown cache id");
    h->caches.erase(it);
    h->states.erase(h->cache_state[cache_id]);
    h->cache_state.erase(cache_id);
  });
}

static SamplingCache& get_cache(sps_handle* h, int id) {
  auto it = h->caches.find(id);
  if (it == h->caches.end()) throw Error(SPS_ERR_STATE, "unknown cache id");
  return it->second;
}

int sps_sample(sps_handle* h, int32_t cache_id, const double* uniforms, int32_t* configuration,
               sps_sample_report* report) {
  return guarded(h, [&] {
    if (!uniforms) throw Error(SPS_ERR_ARGUMENT, "an explicit RNG is required");
    SamplingCache& c = get_cache(h, cache_id);
    SampleResult r = sample_configuration(*h->E, c, uniforms, nullptr);
    if (configuration)
      for (size_t i = 0; i < r.config.size(); ++i) configuration[i] = r.config[i];
    if (report) fill_sample(r, *report);
  });
}

int sps_sample_conditionals(sps_handle* h, int32_t cache_id, const double* uniforms, const int32_t* given,
                            int32_t* configuration, double* conditionals, sps_sample_report* report) {
  return guarded(h, [&] {
    if (!uniforms && !given) throw Error(SPS_ERR_ARGUMENT, "an explicit RNG is required");
    SamplingCache& c = get_cache(h, cache_id);
    std::vector<int> cfg;
    if (given) cfg.assign(given, given + c.Lx * c.Ly);
    SampleResult r = sample_configuration(*h->E, c, given ? nullptr : uniforms, given ? cfg.data() : nullptr);
    if (configuration)
      for (size_t i = 0; i < r.config.size(); ++i) configuration[i] = r.config[i];
    if (conditionals) {
      // r.conditionals follow the draw order; the diagonal draw visits the
      // sites by anti-diagonals
      std::vector<int> order;
      if (c.method.diagonal) order = diagonal_draw_order(c.Lx, c.Ly);
      for (size_t i = 0; i < r.config.size(); ++i) conditionals[i] = 0.0;
      for (size_t i = 0; i < r.conditionals.size() && i < r.config.size(); ++i)
        conditionals[c.method.diagonal ? order[i] : (int)i] = r.conditionals[i];
    }
    if (report) fill_sample(r, *report);
  });
}

int sps_sample_probability(sps_handle* h, int32_t cache_id, const int32_t* configuration,
                           sps_sample_report* report) {
  return guarded(h, [&] {
    if (!configuration) throw Error(SPS_ERR_ARGUMENT, "missing configuration");
    SamplingCache& c = get_cache(h, cache_id);
    std::vector<int> cfg(configuration, configuration + c.Lx * c.Ly);
    SampleResult r = sample_configuration(*h->E, c, nullptr, cfg.data());
    if (report) fill_sample(r, *report);
  });
}

int sps_sample_batch(sps_handle* h, int32_t cache_id, int32_t n, const double* uniforms, int32_t* configurations,
                     double* log_probabilities, sps_sample_report* reports) {
  return guarded(h, [&] {
    if (n > 0 && (!uniforms || !configurations || !log_probabilities))
      throw Error(SPS_ERR_ARGUMENT, "missing batch buffers");
    SamplingCache& c = get_cache(h, cache_id);
    const int L = c.Lx * c.Ly;
    // the shared cache is read-only
    run_batch(h, n, [&](Engine& E, int i) {
      SampleResult r = sample_configuration(E, c, uniforms + (size_t)i * L, nullptr);
      for (int k = 0; k < L; ++k) configurations[(size_t)i * L + k] = r.config[k];
      log_probabilities[i] = r.log_probability;
      if (reports) fill_sample(r, reports[i]);
    });
  });
}

int sps_sample_probability_batch(sps_handle* h, int32_t cache_id, int32_t n, const int32_t* configurations,
                                 double* log_probabilities, sps_sample_report* reports) {
  return guarded(h, [&] {
    if (n > 0 && (!configurations || !log_probabilities)) throw Error(SPS_ERR_ARGUMENT, "missing batch buffers");
    SamplingCache& c = get_cache(h, cache_id);
    const int L = c.Lx * c.Ly;
    run_batch(h, n, [&](Engine& E, int i) {
      std::vector<int> cfg(configurations + (size_t)i * L, configurations + (size_t)(i + 1) * L);
      SampleResult r = sample_configuration(E, c, nullptr, cfg.data());
      log_probabilities[i] = r.log_probability;
      if (reports) fill_sample(r, reports[i]);
    });
  });
}

int sps_project(sps_handle* h, int32_t pepo_id, const int32_t* configuration, int32_t* state_id,
                double* log_normalizations) {
  return guarded(h, [&] {
    State& p = get_state(h, pepo_id);
    std::vector<int> cfg(configuration, configuration + p.Lx * p.Ly);
    std::vector<double> ln;
    State s = project_configuration(*h->E, p, cfg.data(), &ln);
    int id = h->next_id++;
    h->states[id] = std::move(s);
    *state_id = id;
    if (log_normalizations) std::memcpy(log_normalizations, ln.data(), ln.size() * sizeof(double));
  });
}

int sps_project_batch(sps_handle* h, int32_t pepo_id, int32_t n, const int32_t* configurations, int32_t* state_ids,
                      double* log_normalizations) {
  return guarded(h, [&] {
    State& p = get_state(h, pepo_id);
    if (n > 0 && (!configurations || !state_ids)) throw Error(SPS_ERR_ARGUMENT, "missing batch buffers");
    const size_t L = (size_t)p.Lx * p.Ly;
    std::vector<State> out(std::max(n, 0));
    run_batch(h, n, [&](Engine& E, int i) {
      std::vector<int> cfg(configurations + i * L, configurations + (i + 1) * L);
      std::vector<double> ln;
      out[i] = project_configuration(E, p, cfg.data(), &ln);
      if (log_normalizations) std::memcpy(log_normalizations + i * L, ln.data(), ln.size() * sizeof(double));
    });
    for (int i = 0; i < n; ++i) {
      int id = h->next_id++;
      h->states[id] = std::move(out[i]);
      state_ids[i] = id;
    }
  });
}

}  // extern "C"
