// Serving loop for many independent CP-stream sessions.
//
// The reference processes one stream's slices one at a time
// (src/streaming_cpd.cpp:26-366); it has no server.  Here a server accepts
// slice updates for many streams of different shapes and ranks, keeps each
// stream's model, Grams and ADMM state resident on the device, admits
// streams under an HBM budget, and overlaps the streams' work on the device:
//
//   * W worker threads, each with its own non-blocking CUDA stream; a
//     worker takes the next stream that has queued slices and is not being
//     processed, runs one slice update on its CUDA stream, and puts the
//     stream back if it has more work -- so requests that arrive while
//     others run are picked up as soon as a worker frees up, and the
//     updates of different streams run concurrently on the GPU;
//   * a stream's slices run in arrival order, one at a time (its state is
//     sequential);
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

#include "alto_internal.cuh"

namespace alto {
void stream_set_cuda_stream(alto_stream_session* s, cudaStream_t st);
}

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
  std::unordered_map<uint64_t, TicketInfo> tickets;
  // latencies of the last kLatencyWindow completed slices (a ring)
  std::vector<double> lat_ms;
  size_t lat_next = 0;
  uint64_t submitted = 0, completed = 0;
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

void worker_main(alto_server* s) {
  cudaSetDevice(s->device);
  cudaStream_t cs = nullptr;
  cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  tls_alloc_stream = cs;
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_work.wait(lk, [&] { return s->stop || !s->ready.empty(); });
    if (s->ready.empty()) break;  // stop requested and nothing left
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
    if (st == ALTO_OK && !r->sess) {
      const alto_stream_config& c = r->cfg;
      st = alto_stream_open(c.nmodes, c.stream_mode, c.rank, c.constraint, c.forgetting, c.max_inner_iters,
                            c.epsilon, cs, &r->sess);
      if (st == ALTO_OK) st = alto_stream_set_model(r->sess, c.model);
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
      st = alto_stream_push(r->sess, &coo, q->init.data(), q->init.size(), &inner);
    }
    const double t_end = now_s();

    lk.lock();
    s->busy_workers--;
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
      s->ready.push_back(sid);
      s->cv_work.notify_one();
    }
    delete q;
    s->cv_done.notify_all();
  }
  lk.unlock();
  tls_alloc_stream = nullptr;
  cudaStreamSynchronize(cs);
  cudaStreamDestroy(cs);
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
  }
  for (auto& w : s->workers) w.join();
  for (auto& kv : s->streams) {
    for (SliceReq* q : kv.second->q) delete q;
    if (kv.second->sess) alto_stream_close(kv.second->sess);
    delete kv.second;
  }
  delete s;
  return ALTO_OK;
}

}  // extern "C"
