// Host loops over the C ABI: the continuous-batching server (ar_server_run) and the
// autotuner's candidate timing (ar_tune_candidates).  No counterpart in the reference, which
// steps one scene per frame with fixed settings.
//
// Per round of the loop: requests whose arrival time has passed join the waiting queue;
// waiting requests are admitted in arrival order while they fit (HBM budget by
// ar_scene_footprint, AR_MAX_BATCH_* and the particle cap), each as a clone of its resident
// template on the admission stream; copies the host can see completed retire their requests
// and free their budget; then one tick is queued on the compute stream (member list with step
// budgets when it changed, tick_steps batch steps, the finished scenes' state copies and an
// event).  The host never waits for the tick it has just queued, only for the oldest one when
// max_inflight ticks are in flight, so admission overlaps device work.
#include <algorithm>
#include <chrono>
#include <deque>
#include <thread>
#include <vector>

#include "ar_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

struct Template {
  ar_scene* proto = nullptr;
  size_t bytes = 0;     // ar_scene_footprint
  uint64_t cells = 0;   // ar_scene_cells
  int n = 0, nb = 0;
};

struct Need {
  double bytes = 0;
  uint64_t cells = 0;
  long long particles = 0;
};

struct Active {
  int req;
  ar_scene* scene;
  long long left;  // steps still to run
  Need need;
};

struct Retiring {
  int req;
  Need need;
  cudaEvent_t done;
};

}  // namespace

struct ar_server {
  ar_ctx* ctx = nullptr;
  double budget = 0;
  int tick_steps = 10;
  long long max_particles = AR_MAX_BATCH_PARTICLES;
  int max_inflight = 2;
  std::vector<Template> templates;
  ar_batch* batch = nullptr;
  cudaStream_t stream = nullptr, adm = nullptr;
  float* scratch = nullptr;  // pinned, for the state copies nobody keeps
  size_t scratch_bytes = 0;
  std::vector<cudaEvent_t> spare_events;

  cudaEvent_t event() {
    cudaEvent_t e = nullptr;
    if (!spare_events.empty()) {
      e = spare_events.back();
      spare_events.pop_back();
    } else if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return e;
  }
  void recycle(cudaEvent_t e) {
    if (e) spare_events.push_back(e);
  }
};

extern "C" {

ar_status ar_server_create(ar_ctx* ctx, double hbm_budget_bytes, int tick_steps,
                           long long max_batch_particles, int max_inflight, ar_server** out) {
  if (!ctx || !out || !(hbm_budget_bytes > 0) || tick_steps <= 0) return AR_ERR_INVALID_ARG;
  *out = nullptr;
  ar_server* s = new ar_server();
  s->ctx = ctx;
  s->budget = hbm_budget_bytes;
  s->tick_steps = tick_steps;
  s->max_particles = max_batch_particles > 0
                         ? std::min<long long>(max_batch_particles, AR_MAX_BATCH_PARTICLES)
                         : AR_MAX_BATCH_PARTICLES;
  s->max_inflight = std::max(1, max_inflight);
  ar_status st = ar_batch_create(ctx, &s->batch);
  if (st == AR_OK &&
      (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
       cudaStreamCreateWithFlags(&s->adm, cudaStreamNonBlocking) != cudaSuccess)) {
    cudaGetLastError();
    arh::set_error("ar_server_create: stream creation failed");
    st = AR_ERR_CUDA;
  }
  if (st != AR_OK) {
    ar_server_destroy(s);
    return st;
  }
  *out = s;
  return AR_OK;
}

ar_status ar_server_add_template(ar_server* s, const ar_scene_desc* desc,
                                 const ar_scene_init* init, int* id) {
  if (!s || !desc || !init || !id) return AR_ERR_INVALID_ARG;
  Template t;
  ar_status st = ar_scene_create(s->ctx, desc, init, reinterpret_cast<ar_stream_t>(s->adm),
                                 &t.proto);
  if (st != AR_OK) return st;
  t.bytes = ar_scene_footprint(desc);
  t.cells = ar_scene_cells(desc);
  t.n = desc->num_particles;
  t.nb = desc->num_bodies;
  const size_t need = 16 * sizeof(float) * (size_t)t.nb;
  if (need > s->scratch_bytes) {
    if (s->scratch) cudaFreeHost(s->scratch);
    s->scratch = nullptr;
    s->scratch_bytes = 0;
    if (cudaMallocHost((void**)&s->scratch, need) != cudaSuccess) {
      cudaGetLastError();
      ar_scene_destroy(t.proto);
      arh::set_error("ar_server_add_template: pinned scratch allocation failed");
      return AR_ERR_OOM;
    }
    s->scratch_bytes = need;
  }
  *id = (int)s->templates.size();
  s->templates.push_back(t);
  return AR_OK;
}

ar_status ar_server_run(ar_server* s, int n, const int* template_id, const int* steps,
                        const double* arrival_s, double time_limit_s, float* const* h_results,
                        double* latency_s, ar_server_stats* stats) {
  if (!s || n < 0 || (n > 0 && (!template_id || !steps || !arrival_s || !latency_s)))
    return AR_ERR_INVALID_ARG;
  for (int i = 0; i < n; ++i) {
    if (template_id[i] < 0 || template_id[i] >= (int)s->templates.size() || steps[i] < 0) {
      arh::set_error("ar_server_run: request %d names no template or a negative K", i);
      return AR_ERR_INVALID_ARG;
    }
    latency_s[i] = -1.0;
  }
  // the templates' uploads are done before the clock starts
  if (cudaStreamSynchronize(s->adm) != cudaSuccess) return arh::check_launch("ar_server_run");
  ar_server_stats out{};
  out.offered = n;
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return arrival_s[a] < arrival_s[b]; });
  size_t next = 0;  // next request of `order` to arrive
  std::deque<int> waiting;
  std::vector<Active> active;
  std::vector<Retiring> retiring;
  std::vector<ar_scene*> leaving;   // finished scenes still members of the batch
  std::deque<cudaEvent_t> inflight;  // queued ticks, oldest first
  Need used;
  bool changed = false;
  ar_status status = AR_OK;
  const cudaStream_t st = s->stream;
  const ar_stream_t sth = reinterpret_cast<ar_stream_t>(st);
  auto fits = [&](const Need& a) {
    return used.bytes + a.bytes <= s->budget && used.cells + a.cells <= AR_MAX_BATCH_CELLS &&
           used.particles + a.particles <= s->max_particles;
  };
  auto drop_leaving = [&]() {
    for (ar_scene* g : leaving) ar_scene_destroy_async(g, sth);
    leaving.clear();
  };
  const Clock::time_point t0 = Clock::now();
  while (status == AR_OK &&
         (next < order.size() || !waiting.empty() || !active.empty() || !retiring.empty())) {
    const double now = seconds_since(t0);
    while (next < order.size() && arrival_s[order[next]] <= now) waiting.push_back(order[next++]);
    // ---- admission (overlaps the ticks in flight) ----
    const Clock::time_point ta = Clock::now();
    bool admitted = false;
    while (!waiting.empty() && (time_limit_s < 0 || now <= time_limit_s)) {
      const int r = waiting.front();
      const Template& t = s->templates[template_id[r]];
      const Need need{(double)t.bytes, t.cells, t.n};
      if (!fits(need)) {
        if (!active.empty() || !retiring.empty()) break;  // wait for resident scenes to leave
        if (need.cells > AR_MAX_BATCH_CELLS || need.particles > s->max_particles) {
          arh::set_error("ar_server_run: request %d can never be admitted", r);
          status = AR_ERR_INVALID_ARG;
          break;
        }
      }
      waiting.pop_front();
      ar_scene* g = nullptr;
      status = ar_scene_clone_async(t.proto, reinterpret_cast<ar_stream_t>(s->adm), &g);
      if (status != AR_OK) break;
      active.push_back(Active{r, g, steps[r], need});
      used.bytes += need.bytes;
      used.cells += need.cells;
      used.particles += need.particles;
      admitted = changed = true;
    }
    if (admitted) {
      cudaEvent_t e = s->event();
      cudaEventRecord(e, s->adm);
      cudaStreamWaitEvent(st, e, 0);
      s->recycle(e);  // a recorded event may be re-recorded once waited on
    }
    out.host_admit_s += seconds_since(ta);
    if (status != AR_OK) break;
    // ---- retire: finished copies the host can see ----
    const Clock::time_point tr = Clock::now();
    for (size_t i = 0; i < retiring.size();) {
      if (cudaEventQuery(retiring[i].done) == cudaSuccess) {
        const Retiring& x = retiring[i];
        latency_s[x.req] = seconds_since(t0) - arrival_s[x.req];
        used.bytes -= x.need.bytes;
        used.cells -= x.need.cells;
        used.particles -= x.need.particles;
        ++out.completed;
        s->recycle(x.done);
        retiring.erase(retiring.begin() + (long)i);
      } else {
        ++i;
      }
    }
    out.host_retire_s += seconds_since(tr);
    if (active.empty()) {
      const Clock::time_point tw = Clock::now();
      if (!retiring.empty()) {  // nothing to step: wait for the oldest copy
        cudaEventSynchronize(retiring.front().done);
      } else if (next < order.size()) {  // idle until the next arrival (at most 1 ms)
        const double wait = std::min(0.001, arrival_s[order[next]] - seconds_since(t0));
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
      } else if (time_limit_s >= 0 && now > time_limit_s) {
        break;  // the rest can no longer be admitted
      }
      out.host_wait_s += seconds_since(tw);
      if (!leaving.empty()) {
        status = ar_batch_set_scenes(s->batch, nullptr, 0);
        drop_leaving();
      }
      continue;
    }
    // ---- queue one tick ----
    const Clock::time_point tb = Clock::now();
    if (changed || out.ticks == 0) {
      std::vector<ar_scene*> members(active.size());
      std::vector<int64_t> left(active.size());
      for (size_t i = 0; i < active.size(); ++i) {
        members[i] = active[i].scene;
        left[i] = active[i].left;
      }
      status = ar_batch_set_scenes_limited(s->batch, members.data(), (int)members.size(),
                                           left.data());
      changed = false;
      drop_leaving();  // no longer members: freed behind the ticks that used them
    }
    out.host_set_s += seconds_since(tb);
    if (status != AR_OK) break;
    const Clock::time_point tw = Clock::now();
    while ((int)inflight.size() >= s->max_inflight) {
      cudaEventSynchronize(inflight.front());
      s->recycle(inflight.front());
      inflight.pop_front();
    }
    out.host_wait_s += seconds_since(tw);
    const Clock::time_point tc = Clock::now();
    const int k = s->tick_steps;
    status = ar_batch_step(s->ctx, s->batch, k, 1, sth);
    if (status != AR_OK) break;
    ++out.ticks;
    out.peak_resident = std::max(out.peak_resident, (int)active.size());
    out.peak_bytes = std::max(out.peak_bytes, (size_t)used.bytes);
    bool finished = false;
    for (Active& a : active) {
      const long long ran = std::min<long long>(k, a.left);
      out.scene_steps += ran;
      out.particle_steps += ran * a.need.particles;
      a.left -= k;
      if (a.left <= 0) {  // frozen on the device after exactly K steps
        float* dst = h_results && h_results[a.req] ? h_results[a.req] : s->scratch;
        status = ar_scene_download_state_async(a.scene, dst, sth);
        cudaEvent_t e = s->event();
        cudaEventRecord(e, st);
        retiring.push_back(Retiring{a.req, a.need, e});
        leaving.push_back(a.scene);
        finished = true;
      }
    }
    if (finished) {
      active.erase(std::remove_if(active.begin(), active.end(),
                                  [](const Active& a) { return a.left <= 0; }),
                   active.end());
      changed = true;
    }
    cudaEvent_t e = s->event();
    cudaEventRecord(e, st);
    inflight.push_back(e);
    out.host_step_s += seconds_since(tc);
  }
  // drain: every scene still resident leaves the batch and is freed
  if (!leaving.empty() || !active.empty()) {
    ar_batch_set_scenes(s->batch, nullptr, 0);
    for (Active& a : active) leaving.push_back(a.scene);
    drop_leaving();
  }
  cudaStreamSynchronize(st);
  for (Retiring& x : retiring) {
    if (status == AR_OK && cudaEventQuery(x.done) == cudaSuccess) {
      latency_s[x.req] = seconds_since(t0) - arrival_s[x.req];
      ++out.completed;
    }
    s->recycle(x.done);
  }
  for (cudaEvent_t ev : inflight) s->recycle(ev);
  out.wall_s = seconds_since(t0);
  if (stats) *stats = out;
  if (status != AR_OK) return status;
  return ar_ctx_status(s->ctx, sth);
}

ar_status ar_tune_candidates(ar_ctx* ctx, const ar_scene_desc* descs, int n_cand,
                            const ar_scene_init* init, int warmup, int steps, float* ms_per_step) {
  if (!ctx || !descs || !init || !ms_per_step || n_cand < 0 || warmup < 0 || steps <= 0)
    return AR_ERR_INVALID_ARG;
  cudaStream_t st = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    cudaGetLastError();
    if (st) cudaStreamDestroy(st);
    if (a) cudaEventDestroy(a);
    arh::set_error("ar_tune_candidates: stream or event creation failed");
    return AR_ERR_CUDA;
  }
  const ar_stream_t sh = reinterpret_cast<ar_stream_t>(st);
  ar_status status = AR_OK;
  for (int i = 0; i < n_cand && status == AR_OK; ++i) {
    ar_scene* g = nullptr;
    status = ar_scene_create(ctx, &descs[i], init, sh, &g);
    if (status != AR_OK) break;
    // the same scene under candidate i: warm-up steps (graph capture included), then the timed
    // graph replays between two events on the stream
    status = ar_step(ctx, g, warmup, 1, sh);
    if (status == AR_OK) {
      cudaEventRecord(a, st);
      status = ar_step(ctx, g, steps, 1, sh);
      cudaEventRecord(b, st);
    }
    if (status == AR_OK && cudaEventSynchronize(b) == cudaSuccess) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      ms_per_step[i] = ms / (float)steps;
      status = ar_ctx_status(ctx, sh);
    } else if (status == AR_OK) {
      status = arh::check_launch("ar_tune_candidates");
    }
    ar_scene_destroy(g);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(st);
  return status;
}

ar_status ar_server_destroy(ar_server* s) {
  if (!s) return AR_ERR_INVALID_ARG;
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->adm) cudaStreamSynchronize(s->adm);
  if (s->batch) ar_batch_destroy(s->batch);
  for (Template& t : s->templates)
    if (t.proto) ar_scene_destroy(t.proto);
  for (cudaEvent_t e : s->spare_events) cudaEventDestroy(e);
  if (s->scratch) cudaFreeHost(s->scratch);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->adm) cudaStreamDestroy(s->adm);
  delete s;
  return AR_OK;
}

}  // extern "C"
