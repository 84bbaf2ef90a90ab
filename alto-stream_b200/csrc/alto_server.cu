// Serving loop for many independent CP-stream sessions.
//
// The reference processes one stream's slices one at a time
// (src/streaming_cpd.cpp:26-366); it has no server.  Here a server accepts
// slice updates for many streams of different shapes and ranks, keeps each
// stream's model, Grams and ADMM state resident on the device, admits
// streams under an HBM budget, and batches their work on the device:
//
//   * W worker threads, each with its own non-blocking CUDA stream, take
//     the next stream that has a queued slice and is idle and prepare the
//     slice (grow the model, encode the slice, Grams: everything before the
//     inner iterations);
//   * one scheduler thread runs the inner iterations of the prepared slices
//     in stream groups (one per rank and line format, up to kGroupSlots
//     slices each): every step is one inner iteration of every slice in the
//     group, one launch of the group's captured graph, in which each kernel
//     covers all the group's slices.  Between steps, slices whose batch has
//     converged leave (a worker then finishes them: forgetting, previous
//     model, time rows) and newly prepared slices join -- continuous
//     batching at the granularity of one inner iteration;
//   * slices of streams that cannot run grouped (the spCP-stream model,
//     other ranks) run their whole update on the worker;
//   * a stream's slices run in arrival order, one at a time (its state is
//     sequential); a stream's result is bit-identical alone, in any mix, and
//     on the plain one-slice-at-a-time path (alto_stream_push runs a
//     session in a group of one), since each session's arithmetic in a group
//     is that of its own launches;
//   * admission: a stream reserves an estimate of its device footprint from
//     its largest dims and slice size; streams that do not fit the budget
//     wait (their slices queue) until earlier streams close;
//   * latency of every slice is measured from submission to completion.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "alto_group.cuh"

using namespace alto;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SliceReq {
  uint64_t ticket = 0;
  int nmodes = 0;
  std::vector<uint64_t> dims;
  std::vector<std::vector<uint64_t>> cidx;
  std::vector<double> vals;
  std::vector<double> init;
  double t_submit = 0;
};

struct StreamRec {
  int sid = 0;
  alto_stream_config cfg{};
  alto_stream_session* sess = nullptr;
  uint64_t reserve = 0;
  bool admitted = false, busy = false, in_ready = false;
  std::deque<SliceReq*> q;
  alto_status err = ALTO_OK;
  uint64_t done = 0;
  SliceReq* cur = nullptr;            // the slice in the group's hands
  cudaEvent_t ready_ev = nullptr;     // its preparation done (worker stream)
  cudaEvent_t ran_ev = nullptr;       // its inner iterations done (group stream)
};

// Slices per stream group.
constexpr int kGroupSlots = 32;
// Inner iterations per group launch (one: slices join and leave between
// every two iterations).
constexpr int kStepsPerLaunch = 1;

struct GroupRun {
  StreamGroup* g = nullptr;
  cudaStream_t st = nullptr;
  std::vector<StreamRec*> members;
};

struct TicketInfo {
  bool done = false;
  int inner = 0;
  alto_status status = ALTO_OK;
  double latency_ms = 0;
};

}  // namespace

struct alto_server {
  uint64_t budget = 0, reserved = 0;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::unordered_map<int, StreamRec*> streams;
  int next_sid = 1;
  uint64_t next_ticket = 1;
  std::deque<int> ready;    // admitted streams with queued slices, not busy
  std::deque<int> pending;  // streams waiting for admission
  std::vector<std::thread> workers;
  bool stop = false;
  // tickets not yet handed back as done by wait/poll (erased then, so the
  // map holds only outstanding work)
  bool sched_done = false;    // the scheduler has left (set once stopping)
  std::deque<int> finishing;  // streams whose grouped slice has run (a worker finishes it)
  std::deque<int> prepared;   // streams whose slice is prepared (the scheduler groups it)
  std::condition_variable cv_sched;
  std::thread scheduler;
  std::vector<GroupRun> groups;  // used by the scheduler thread only
  std::unordered_map<uint64_t, TicketInfo> tickets;
  // latencies of the last kLatencyWindow completed slices (a ring)
  std::vector<double> lat_ms;
  size_t lat_next = 0;
  uint64_t submitted = 0, completed = 0;
  double prepare_ms = 0, step_ms = 0, finish_ms = 0;
  uint64_t steps = 0, step_slices = 0;
  double t_first = 0, t_last = 0;
  int busy_workers = 0;
};

namespace {

constexpr size_t kLatencyWindow = size_t(1) << 20;

void record_latency(alto_server* s, double ms) {  // caller holds s->mu
  if (s->lat_ms.size() < kLatencyWindow) {
    s->lat_ms.push_back(ms);
  } else {
    s->lat_ms[s->lat_next] = ms;
    s->lat_next = (s->lat_next + 1) % kLatencyWindow;
  }
}

// Device footprint estimate of a stream: model, previous model and duals
// (with growth headroom), the float64 solve buffers, the encoded slice, its
// sort scratch and one row-sorted copy per mode.
uint64_t reserve_estimate(const alto_stream_config& c, const uint64_t* max_dims, uint64_t max_nnz) {
  uint64_t sum_dims = 0, max_dim = 0;
  for (int m = 0; m < c.nmodes; ++m) {
    sum_dims += max_dims[m];
    max_dim = std::max(max_dim, max_dims[m]);
  }
  const uint64_t R = (uint64_t)c.rank;
  const uint64_t model = (sum_dims * R * (4 + 4 + 8) * 3) / 2;
  const uint64_t solve = max_dim * R * (4 + 8 * 4);
  const uint64_t tensor = max_nnz * (16 + 4 + 40 + 8ull * c.nmodes + 8 + 16ull * c.nmodes);
  return model + solve + tensor + (64ull << 10) * c.nmodes + (16ull << 20);
}

void admit_pending(alto_server* s) {  // caller holds s->mu
  while (!s->pending.empty()) {
    StreamRec* r = s->streams[s->pending.front()];
    if (s->reserved + r->reserve > s->budget && s->reserved > 0) break;
    s->pending.pop_front();
    r->admitted = true;
    s->reserved += r->reserve;
    if (!r->q.empty() && !r->busy && !r->in_ready) {
      r->in_ready = true;
      s->ready.push_back(r->sid);
    }
  }
  s->cv_work.notify_all();
}

// Completes a slice: its ticket, the latency record, and the stream's next
// slice made ready (caller holds s->mu).
void complete_slice(alto_server* s, StreamRec* r, SliceReq* q, alto_status st, int inner) {
  const double t_end = now_s();
  TicketInfo& ti = s->tickets[q->ticket];
  ti.done = true;
  ti.inner = inner;
  ti.status = st;
  ti.latency_ms = (t_end - q->t_submit) * 1e3;
  if (st != ALTO_OK) r->err = st;
  record_latency(s, ti.latency_ms);
  s->completed++;
  s->t_last = t_end;
  r->done++;
  r->busy = false;
  if (!r->q.empty()) {
    r->in_ready = true;
    s->ready.push_back(r->sid);
    s->cv_work.notify_one();
  }
  delete q;
  s->cv_done.notify_all();
}

void worker_main(alto_server* s) {
  cudaSetDevice(s->device);
  cudaStream_t cs = nullptr;
  cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  tls_alloc_stream = cs;
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_work.wait(lk, [&] {
      return !s->finishing.empty() || !s->ready.empty() || (s->stop && s->sched_done);
    });
    if (!s->finishing.empty()) {  // a grouped slice has run: finish it
      StreamRec* r = s->streams[s->finishing.front()];
      s->finishing.pop_front();
      SliceReq* q = r->cur;
      r->cur = nullptr;
      s->busy_workers++;
      lk.unlock();
      int inner = 0;
      const double t0 = now_s();
      alto_status st = cuda_status(cudaStreamWaitEvent(cs, r->ran_ev, 0), "cudaStreamWaitEvent", __FILE__, __LINE__);
      if (st == ALTO_OK) {
        stream_set_cuda_stream(r->sess, cs);
        st = stream_finish_grouped(r->sess, &inner);
      }
      lk.lock();
      s->finish_ms += (now_s() - t0) * 1e3;
      s->busy_workers--;
      complete_slice(s, r, q, st, inner);
      continue;
    }
    if (s->ready.empty()) break;  // stopping, and nothing left
    const int sid = s->ready.front();
    s->ready.pop_front();
    StreamRec* r = s->streams[sid];
    r->in_ready = false;
    r->busy = true;
    SliceReq* q = r->q.front();
    r->q.pop_front();
    s->busy_workers++;
    lk.unlock();

    alto_status st = r->err;
    int inner = 0;
    bool grouped = false;
    const double t_prep = now_s();
    if (st == ALTO_OK && !r->sess) {
      const alto_stream_config& c = r->cfg;
      st = alto_stream_open(c.nmodes, c.stream_mode, c.rank, c.constraint, c.forgetting, c.max_inner_iters,
                            c.epsilon, cs, &r->sess);
      if (st == ALTO_OK) st = alto_stream_set_model(r->sess, c.model);
      if (st == ALTO_OK &&
          (cudaEventCreateWithFlags(&r->ready_ev, cudaEventDisableTiming) != cudaSuccess ||
           cudaEventCreateWithFlags(&r->ran_ev, cudaEventDisableTiming) != cudaSuccess))
        st = cuda_status(cudaGetLastError(), "cudaEventCreate", __FILE__, __LINE__);
    }
    if (st == ALTO_OK) {
      stream_set_cuda_stream(r->sess, cs);
      std::vector<const void*> ptrs(q->nmodes);
      for (int m = 0; m < q->nmodes; ++m) ptrs[m] = q->cidx[m].data();
      alto_coo coo;
      coo.nmodes = q->nmodes;
      coo.dims = q->dims.data();
      coo.nnz = q->vals.size();
      coo.cidx = ptrs.data();
      coo.index_bytes = 8;
      coo.vals = q->vals.data();
      coo.val_dtype = ALTO_F64;
      coo.on_device = 0;
      st = stream_prepare_grouped(r->sess, &coo, q->init.data(), q->init.size(), &grouped);
      if (st == ALTO_OK && !grouped) st = stream_run_ungrouped(r->sess, &inner);
      if (st == ALTO_OK && grouped)
        st = cuda_status(cudaEventRecord(r->ready_ev, cs), "cudaEventRecord", __FILE__, __LINE__);
    }
    lk.lock();
    s->prepare_ms += (now_s() - t_prep) * 1e3;
    s->busy_workers--;
    if (st == ALTO_OK && grouped) {  // to the scheduler
      r->cur = q;
      s->prepared.push_back(sid);
      s->cv_sched.notify_one();
      continue;
    }
    complete_slice(s, r, q, st, inner);
  }
  lk.unlock();
  tls_alloc_stream = nullptr;
  cudaStreamSynchronize(cs);
  cudaStreamDestroy(cs);
}

// The scheduler: prepared slices join stream groups; every round, one group
// launch per group with members, then the members whose batch is done
// leave and go to the workers to be finished.
void scheduler_main(alto_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  auto busy = [&] {
    for (auto& g : s->groups)
      if (!g.members.empty()) return true;
    return false;
  };
  while (true) {
    s->cv_sched.wait(lk, [&] { return s->stop || !s->prepared.empty() || busy(); });
    if (s->stop && s->prepared.empty() && !busy()) {
      // stop only once the workers have nothing left that could be prepared
      bool idle = s->ready.empty() && s->finishing.empty() && s->busy_workers == 0;
      if (idle) break;
      s->cv_sched.wait_for(lk, std::chrono::milliseconds(5));
      continue;
    }
    std::vector<StreamRec*> joining;
    while (!s->prepared.empty()) {
      joining.push_back(s->streams[s->prepared.front()]);
      s->prepared.pop_front();
    }
    lk.unlock();
    std::vector<std::pair<StreamRec*, alto_status>> failed;
    for (StreamRec* r : joining) {
      GroupRun* gr = nullptr;
      for (auto& g : s->groups)
        if ((int)g.members.size() < kGroupSlots && group_fits(g.g, r->sess)) {
          gr = &g;
          break;
        }
      if (!gr) {
        GroupRun g;
        alto_status st = cuda_status(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking), "cudaStreamCreate",
                                     __FILE__, __LINE__);
        if (st == ALTO_OK) st = group_create(r->sess, kGroupSlots, g.st, &g.g);
        if (st != ALTO_OK) {
          if (g.st) cudaStreamDestroy(g.st);
          failed.emplace_back(r, st);
          continue;
        }
        s->groups.push_back(g);
        gr = &s->groups.back();
      }
      cudaStreamWaitEvent(gr->st, r->ready_ev, 0);
      gr->members.push_back(r);
    }
    const double t_step = now_s();
    uint64_t nsteps = 0, nslices = 0;
    for (auto& g : s->groups) {
      if (g.members.empty()) continue;
      nsteps += 1;
      nslices += g.members.size();
      std::vector<alto_stream_session*> sess;
      for (StreamRec* r : g.members) sess.push_back(r->sess);
      alto_status st = group_set(g.g, sess.data(), (int)sess.size());
      if (st == ALTO_OK) st = group_launch(g.g, kStepsPerLaunch);
      if (st != ALTO_OK) {
        for (StreamRec* r : g.members) failed.emplace_back(r, st);
        g.members.clear();
      }
    }
    std::vector<StreamRec*> done;
    for (auto& g : s->groups) {
      const int k = (int)g.members.size();
      if (!k) continue;
      std::vector<int> running(k, 0);
      alto_status st = group_states(g.g, running.data(), nullptr, nullptr, nullptr);
      std::vector<StreamRec*> keep;
      for (int q = 0; q < k; ++q) {
        StreamRec* r = g.members[q];
        if (st != ALTO_OK) {
          failed.emplace_back(r, st);
        } else if (running[q]) {
          keep.push_back(r);
        } else {
          cudaEventRecord(r->ran_ev, g.st);
          done.push_back(r);
        }
      }
      g.members.swap(keep);
    }
    lk.lock();
    s->step_ms += (now_s() - t_step) * 1e3;
    s->steps += nsteps;
    s->step_slices += nslices;
    for (StreamRec* r : done) {
      s->finishing.push_back(r->sid);
      s->cv_work.notify_one();
    }
    for (auto& f : failed) {
      SliceReq* q = f.first->cur;
      f.first->cur = nullptr;
      complete_slice(s, f.first, q, f.second, 0);
    }
  }
  s->sched_done = true;
  s->cv_work.notify_all();
  lk.unlock();
  for (auto& g : s->groups) {
    group_destroy(g.g);
    cudaStreamDestroy(g.st);
  }
  s->groups.clear();
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = p * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

extern "C" {

alto_status alto_server_create(uint64_t hbm_budget_bytes, int workers, alto_server** out) {
  if (!out || workers < 1 || workers > 256) {
    set_error("bad arguments (workers 1..256)");
    return ALTO_ERR_INVALID;
  }
  *out = nullptr;
  alto_server* s = new (std::nothrow) alto_server();
  if (!s) return ALTO_ERR_NOMEM;
  s->budget = hbm_budget_bytes;
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    set_error("no CUDA device");
    return ALTO_ERR_CUDA;
  }
  for (int w = 0; w < workers; ++w) s->workers.emplace_back(worker_main, s);
  s->scheduler = std::thread(scheduler_main, s);
  *out = s;
  return ALTO_OK;
}

alto_status alto_server_open(alto_server* s, const alto_stream_config* cfg, const uint64_t* max_dims,
                             uint64_t max_slice_nnz, int* sid) {
  if (!s || !cfg || !max_dims || !sid) {
    set_error("bad arguments");
    return ALTO_ERR_INVALID;
  }
  if (cfg->nmodes < 2 || cfg->nmodes > ALTO_MAX_MODES || cfg->stream_mode < 0 ||
      cfg->stream_mode >= cfg->nmodes || cfg->rank < 1 || cfg->rank > 128 || cfg->max_inner_iters < 1 ||
      (cfg->model != ALTO_MODEL_CPSTREAM && cfg->model != ALTO_MODEL_SPCPSTREAM)) {
    set_error("bad stream configuration");
    return ALTO_ERR_INVALID;
  }
  StreamRec* r = new StreamRec();
  r->cfg = *cfg;
  r->reserve = reserve_estimate(*cfg, max_dims, max_slice_nnz);
  std::lock_guard<std::mutex> lk(s->mu);
  r->sid = s->next_sid++;
  s->streams[r->sid] = r;
  s->pending.push_back(r->sid);
  admit_pending(s);
  *sid = r->sid;
  return ALTO_OK;
}

alto_status alto_server_submit(alto_server* s, int sid, const alto_coo* batch, const double* init_vals,
                               uint64_t n_init, uint64_t* ticket) {
  if (!s || !batch || batch->on_device || batch->nnz == 0 || !batch->cidx || !batch->vals || !batch->dims ||
      (batch->index_bytes != 4 && batch->index_bytes != 8) ||
      (batch->val_dtype != ALTO_F32 && batch->val_dtype != ALTO_F64)) {
    set_error("server batches are non-empty host COO tensors (4- or 8-byte indices, float32/64 values)");
    return ALTO_ERR_INVALID;
  }
  SliceReq* q = new SliceReq();
  q->nmodes = batch->nmodes;
  q->dims.assign(batch->dims, batch->dims + batch->nmodes);
  q->cidx.resize(batch->nmodes);
  for (int m = 0; m < batch->nmodes; ++m) {
    if (batch->index_bytes == 8) {
      const uint64_t* c = (const uint64_t*)batch->cidx[m];
      q->cidx[m].assign(c, c + batch->nnz);
    } else {
      const uint32_t* c = (const uint32_t*)batch->cidx[m];
      q->cidx[m].assign(c, c + batch->nnz);
    }
  }
  if (batch->val_dtype == ALTO_F64) {
    const double* v = (const double*)batch->vals;
    q->vals.assign(v, v + batch->nnz);
  } else {
    const float* v = (const float*)batch->vals;
    q->vals.assign(v, v + batch->nnz);
  }
  if (n_init && init_vals) q->init.assign(init_vals, init_vals + n_init);
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->streams.find(sid);
  if (it == s->streams.end()) {
    delete q;
    set_error("unknown stream %d", sid);
    return ALTO_ERR_INVALID;
  }
  StreamRec* r = it->second;
  if (r->cfg.nmodes != batch->nmodes) {
    delete q;
    set_error("batch has %d modes, stream %d", batch->nmodes, r->cfg.nmodes);
    return ALTO_ERR_INVALID;
  }
  q->ticket = s->next_ticket++;
  q->t_submit = now_s();
  if (s->submitted == 0) s->t_first = q->t_submit;
  s->submitted++;
  s->tickets[q->ticket] = TicketInfo();
  r->q.push_back(q);
  if (r->admitted && !r->busy && !r->in_ready) {
    r->in_ready = true;
    s->ready.push_back(sid);
    s->cv_work.notify_one();
  }
  if (ticket) *ticket = q->ticket;
  return ALTO_OK;
}

alto_status alto_server_wait(alto_server* s, uint64_t ticket, int* inner_iters, double* latency_ms) {
  if (!s) {
    set_error("server is NULL");
    return ALTO_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    set_error("unknown ticket %llu", (unsigned long long)ticket);
    return ALTO_ERR_INVALID;
  }
  s->cv_done.wait(lk, [&] {
    auto jt = s->tickets.find(ticket);
    return jt == s->tickets.end() || jt->second.done;
  });
  it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {  // another waiter took it first
    set_error("ticket %llu was already handed back", (unsigned long long)ticket);
    return ALTO_ERR_INVALID;
  }
  const TicketInfo ti = it->second;
  s->tickets.erase(it);
  if (inner_iters) *inner_iters = ti.inner;
  if (latency_ms) *latency_ms = ti.latency_ms;
  return ti.status;
}

alto_status alto_server_poll(alto_server* s, uint64_t ticket, int* done, int* inner_iters, double* latency_ms) {
  if (!s || !done) {
    set_error("server or done is NULL");
    return ALTO_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    set_error("unknown ticket %llu", (unsigned long long)ticket);
    return ALTO_ERR_INVALID;
  }
  *done = it->second.done ? 1 : 0;
  if (!it->second.done) return ALTO_OK;
  const TicketInfo ti = it->second;
  s->tickets.erase(it);
  if (inner_iters) *inner_iters = ti.inner;
  if (latency_ms) *latency_ms = ti.latency_ms;
  return ti.status;
}

alto_status alto_server_drain(alto_server* s) {
  if (!s) {
    set_error("server is NULL");
    return ALTO_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  // every admitted stream idle: nothing queued, nothing running
  s->cv_done.wait(lk, [&] {
    for (auto& kv : s->streams)
      if (kv.second->admitted && (kv.second->busy || !kv.second->q.empty())) return false;
    return true;
  });
  for (auto& kv : s->streams)
    if (kv.second->err != ALTO_OK) return kv.second->err;
  return ALTO_OK;
}

alto_status alto_server_stats(alto_server* s, alto_serving_stats* out) {
  if (!s || !out) {
    set_error("bad arguments");
    return ALTO_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->p50_ms = percentile(s->lat_ms, 0.50);
  out->p99_ms = percentile(s->lat_ms, 0.99);
  out->max_ms = s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end());
  const double span = s->t_last - s->t_first;
  out->slices_per_s = span > 0 ? (double)s->completed / span : 0.0;
  out->reserved_bytes = s->reserved;
  int admitted = 0;
  for (auto& kv : s->streams) admitted += kv.second->admitted ? 1 : 0;
  out->admitted_streams = admitted;
  out->pending_streams = (int)s->pending.size();
  out->prepare_ms = s->prepare_ms;
  out->step_ms = s->step_ms;
  out->finish_ms = s->finish_ms;
  out->steps = s->steps;
  out->step_slices = s->step_slices;
  return ALTO_OK;
}

alto_status alto_server_factor(alto_server* s, int sid, int mode, double* host_out, uint64_t* rows) {
  if (!s) {
    set_error("server is NULL");
    return ALTO_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->streams.find(sid);
  if (it == s->streams.end()) {
    set_error("unknown stream %d", sid);
    return ALTO_ERR_INVALID;
  }
  StreamRec* r = it->second;
  s->cv_done.wait(lk, [&] { return !r->busy && (r->q.empty() || !r->admitted); });
  if (!r->sess) {
    if (rows) *rows = 0;
    return r->err;
  }
  return alto_stream_factor(r->sess, mode, host_out, rows);
}

alto_status alto_server_close(alto_server* s, int sid) {
  if (!s) {
    set_error("server is NULL");
    return ALTO_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->streams.find(sid);
  if (it == s->streams.end()) {
    set_error("unknown stream %d", sid);
    return ALTO_ERR_INVALID;
  }
  StreamRec* r = it->second;
  s->cv_done.wait(lk, [&] { return !r->busy && (r->q.empty() || !r->admitted); });
  // never-admitted work is dropped: its tickets finish with an error so that
  // waiters (already blocked or later) return
  for (SliceReq* q : r->q) {
    TicketInfo& ti = s->tickets[q->ticket];
    ti.done = true;
    ti.status = ALTO_ERR_INVALID;
    delete q;
  }
  const bool dropped = !r->q.empty();
  r->q.clear();
  s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), sid), s->pending.end());
  if (r->admitted) s->reserved -= r->reserve;
  s->streams.erase(it);
  alto_stream_session* sess = r->sess;
  const alto_status err = r->err;
  if (r->ready_ev) cudaEventDestroy(r->ready_ev);
  if (r->ran_ev) cudaEventDestroy(r->ran_ev);
  delete r;
  admit_pending(s);
  if (dropped) s->cv_done.notify_all();
  lk.unlock();
  if (sess) alto_stream_close(sess);
  return err;
}

alto_status alto_server_destroy(alto_server* s) {
  if (!s) return ALTO_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
    s->cv_sched.notify_all();
  }
  if (s->scheduler.joinable()) s->scheduler.join();
  for (auto& w : s->workers) w.join();
  for (auto& kv : s->streams) {
    for (SliceReq* q : kv.second->q) delete q;
    if (kv.second->sess) alto_stream_close(kv.second->sess);
    if (kv.second->ready_ev) cudaEventDestroy(kv.second->ready_ev);
    if (kv.second->ran_ev) cudaEventDestroy(kv.second->ran_ev);
    delete kv.second;
  }
  delete s;
  return ALTO_OK;
}

}  // extern "C"
