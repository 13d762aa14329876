// The serving form: a request loop that admits count queries under a device
// memory budget and batches whatever is queued whenever a slot frees up. No
// counterpart in the reference (one graph per run, main.cpp:76-192); every
// served count equals the query's count through the plain path.
//
// Threads: the caller's threads submit and poll; each slot is one host
// worker thread with its own context (CUDA stream). A free worker takes the
// queued queries from the front while they fit (budget, batch caps), builds
// them as one disjoint-union graph (batch.cu) and counts them in one
// persistent launch, so several slots' batches overlap on the device: one
// copies and sorts while another counts. A query's device bytes are bounded
// by serve_estimate(); the sum over queries in flight never exceeds the
// budget, so admission, not the allocator, decides what runs. No device-side
// waits are involved: every synchronisation is a host wait on a stream.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "xt_internal.cuh"

namespace xt {

using Clock = std::chrono::steady_clock;

// Upper bound of the device bytes held while a query of nv vertices and ne
// edge rows is copied in, built and counted. The builder's largest phases:
// its row sort (8 B/row copied in, 8 B/row union ids for batches, 16 B/row
// of row ends in two sort buffers, 8 B/row of sort scratch: 40 B/row) and
// the in-record sort (the same 16 B/row buffers, plus per unique edge 4 B
// columns, 4 B padded columns and two 8 B record arrays: up to 52 B/row with
// the input and union ids held; 72 B/row with the 16-byte records this
// bound was first written for). Vertex arrays stay below 120 B/vertex
// through the plan. 80 B/row leaves room for CUB's scratch on top of these;
// tests/test_gpu_serve.py checks it against the measured peak.
int64_t serve_estimate(int64_t nv, int64_t ne) {
  if (nv < 0 || ne < 0) return -1;
  return 80 * ne + 120 * nv + (int64_t(4) << 20);
}

struct Query {
  int64_t nv = 0, ne = 0;
  const int32_t *src = nullptr, *dst = nullptr;
  int64_t est = 0;
  xt_status status = XT_ERR_NOT_READY;
  int64_t count = -1;
  Clock::time_point t_submit, t_done;
};

struct Server {
  int device = 0;
  xt_serve_config cfg{};
  std::vector<xt_ctx *> slot_ctx;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work;  // a query queued, budget freed or closing
  std::condition_variable cv_done;  // a result published
  std::deque<int64_t> queue;
  std::unordered_map<int64_t, Query> q;  // by ticket, until its result is taken
  int64_t next_ticket = 1;
  int64_t budget_used = 0;
  bool closing = false;
  xt_serve_stats st{};
  // device bytes all slots' allocations hold together, and at most
  std::atomic<int64_t> dev_live{0}, dev_peak{0};
  Clock::time_point t_open;
  std::deque<xt_serve_batch> log;  // the most recent batches
};

constexpr size_t kLogMax = 65536;

static int64_t ns_since(const Server *S, Clock::time_point t) {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(t - S->t_open).count();
}

struct Result {
  xt_status status;
  int64_t count;
};

struct BatchTimes {
  Clock::time_point built;
  xt_status status = XT_OK;
};

// Builds and counts one batch on slot context c and returns each query's
// result (the queries are only read here: the caller publishes the results
// under the lock).
static std::vector<Result> run_batch(Server *S, Ctx *c, const std::vector<const Query *> &b, BatchTimes *bt) {
  const int64_t ng = int64_t(b.size());
  const int orient = S->cfg.orient;
  std::vector<int64_t> voff(ng + 1, 0), eoff(ng + 1, 0);
  for (int64_t i = 0; i < ng; i++) {
    voff[i + 1] = voff[i] + b[i]->nv;
    eoff[i + 1] = eoff[i] + b[i]->ne;
  }
  const int64_t ne = eoff[ng];
  int32_t *ds = nullptr, *dd = nullptr;
  int64_t *res = nullptr;
  std::vector<int64_t> per(ng + 1, 0);
  Graph g;
  xt_status s = dalloc_n(c, &ds, size_t(ne > 0 ? ne : 1));
  if (s == XT_OK) s = dalloc_n(c, &dd, size_t(ne > 0 ? ne : 1));
  if (s == XT_OK) s = dalloc_n(c, &res, size_t(ng + 1));
  for (int64_t i = 0; i < ng && s == XT_OK; i++) {
    if (b[i]->ne == 0) continue;
    const size_t bytes = sizeof(int32_t) * size_t(b[i]->ne);
    s = cuda_status(c, cudaMemcpyAsync(ds + eoff[i], b[i]->src, bytes, cudaMemcpyHostToDevice, c->stream), "H2D");
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(dd + eoff[i], b[i]->dst, bytes, cudaMemcpyHostToDevice, c->stream), "H2D");
  }
  if (s == XT_OK) {
    if (ng == 1) {
      s = build_from_edges(c, b[0]->nv, b[0]->ne, ds, dd, orient, &g);
      if (s == XT_OK) s = make_plan(&g);  // ends with a host wait on the stream
      bt->built = Clock::now();
      if (s == XT_OK) s = count_graph(&g, res, nullptr, nullptr);
      if (s == XT_OK) s = cuda_status(c, cudaMemcpyAsync(per.data(), res, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                                         c->stream), "D2H");
    } else {
      s = build_batch(c, ng, voff.data(), eoff.data(), ds, dd, orient, &g);
      if (s == XT_OK) s = make_plan(&g);
      bt->built = Clock::now();
      if (s == XT_OK) s = count_graph(&g, res, nullptr, res + 1);
      if (s == XT_OK)
        s = cuda_status(c, cudaMemcpyAsync(per.data(), res, sizeof(int64_t) * size_t(ng + 1),
                                           cudaMemcpyDeviceToHost, c->stream), "D2H");
    }
    if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "count");
  }
  free_graph_device(&g);
  dfree(c, ds);
  dfree(c, dd);
  dfree(c, res);
  cudaStreamSynchronize(c->stream);
  std::vector<Result> out(size_t(ng), Result{s, -1});
  bt->status = s;
  if (ng > 1 && s == XT_ERR_INVALID) {
    // one query's ids are out of range: count each alone so only it fails
    BatchTimes one;
    for (int64_t i = 0; i < ng; i++) out[i] = run_batch(S, c, std::vector<const Query *>{b[i]}, &one)[0];
    return out;
  }
  if (s == XT_OK)
    for (int64_t i = 0; i < ng; i++) out[i].count = ng == 1 ? per[0] : per[i + 1];
  return out;
}

static void worker(Server *S, int slot) {
  cudaSetDevice(S->device);
  Ctx *c = &S->slot_ctx[slot]->c;
  const int64_t max_g = S->cfg.max_batch_graphs, max_e = S->cfg.max_batch_edges;
  while (true) {
    std::vector<Query *> batch;
    int64_t est = 0, batch_edges = 0;
    Clock::time_point t_take;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] {
        if (S->closing) return true;
        if (S->queue.empty()) return false;
        return S->budget_used + S->q[S->queue.front()].est <= S->cfg.budget_bytes;
      });
      if (S->closing) return;
      int64_t edges = 0, verts = 0;
      while (!S->queue.empty() && int64_t(batch.size()) < max_g) {
        Query &x = S->q[S->queue.front()];
        if (S->budget_used + est + x.est > S->cfg.budget_bytes) break;
        // caps: a query larger than max_e still runs, alone; the union stays below 2^31 ids
        if (!batch.empty() && (edges + x.ne > max_e || verts + x.nv >= (int64_t(1) << 31))) break;
        batch.push_back(&x);
        est += x.est;
        edges += x.ne;
        verts += x.nv;
        S->queue.pop_front();
      }
      batch_edges = edges;
      t_take = Clock::now();
      S->budget_used += est;
      if (S->budget_used > S->st.budget_peak) S->st.budget_peak = S->budget_used;
      S->st.queued = int64_t(S->queue.size());
      S->st.in_flight += int64_t(batch.size());
      S->st.batches++;
      if (int64_t(batch.size()) > S->st.max_batch) S->st.max_batch = int64_t(batch.size());
    }
    // unordered_map nodes are stable: the queries stay put while the lock is
    // released, and no other thread writes them or takes them before their
    // status leaves XT_ERR_NOT_READY, which happens under the lock below
    BatchTimes bt;
    bt.built = t_take;
    const std::vector<Result> res = run_batch(S, c, std::vector<const Query *>(batch.begin(), batch.end()), &bt);
    const Clock::time_point now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      xt_serve_batch rec;
      rec.t_take_ns = ns_since(S, t_take);
      rec.t_built_ns = ns_since(S, bt.built);
      rec.t_done_ns = ns_since(S, now);
      rec.graphs = int64_t(batch.size());
      rec.edge_rows = batch_edges;
      rec.slot = slot;
      rec.status = bt.status;
      S->log.push_back(rec);
      if (S->log.size() > kLogMax) S->log.pop_front();
      for (size_t i = 0; i < batch.size(); i++) {
        Query *x = batch[i];
        x->status = res[i].status;
        x->count = res[i].count;
        x->t_done = now;
        if (x->status == XT_OK) S->st.completed++;
        else S->st.failed++;
      }
      S->budget_used -= est;
      S->st.in_flight -= int64_t(batch.size());
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
  }
}

}  // namespace xt

struct xt_server {
  xt::Server s;
};

using namespace xt;

extern "C" {

int64_t xt_serve_estimate(int64_t nv, int64_t ne) { return serve_estimate(nv, ne); }

xt_status xt_serve_open(int device, const xt_serve_config *cfg, xt_server **out) {
  if (!out) return XT_ERR_INVALID;
  *out = nullptr;
  xt_serve_config c{};
  if (cfg) c = *cfg;
  if (c.orient != XT_ORIENT_ID && c.orient != XT_ORIENT_DEGREE) return XT_ERR_INVALID;
  if (c.budget_bytes <= 0) c.budget_bytes = int64_t(150) << 30;
  if (c.max_batch_graphs <= 0) c.max_batch_graphs = 4096;
  if (c.max_batch_edges <= 0) c.max_batch_edges = int64_t(1) << 26;
  if (c.slots <= 0) c.slots = 3;
  if (c.slots > 64) return XT_ERR_INVALID;
  xt_ctx *probe = nullptr;
  XT_TRY(xt_open(device, &probe));  // device checks (and XT_ERR_NO_DEVICE) as for a context
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
    const int64_t cap = int64_t(free_b) - (int64_t(2) << 30);
    if (cap > 0 && c.budget_bytes > cap) c.budget_bytes = cap;
  }
  xt_close(probe);
  xt_server *srv = new (std::nothrow) xt_server();
  if (!srv) return XT_ERR_OOM;
  Server *S = &srv->s;
  S->device = device;
  S->cfg = c;
  S->st.budget_bytes = c.budget_bytes;
  S->t_open = Clock::now();
  for (int i = 0; i < c.slots; i++) {
    xt_ctx *sc = nullptr;
    xt_status s = xt_open(device, &sc);
    if (s != XT_OK) {
      for (xt_ctx *o : S->slot_ctx) xt_close(o);
      delete srv;
      return s;
    }
    sc->c.shared_live = &S->dev_live;
    sc->c.shared_peak = &S->dev_peak;
    S->slot_ctx.push_back(sc);
  }
  // Grow the device's stream-ordered pool once, up to what the slots' largest
  // batches hold together: growing it while queries run stalls them (mapping
  // fresh memory), and the pool keeps freed memory (release threshold max).
  {
    int64_t want = std::min<int64_t>(c.budget_bytes, int64_t(c.slots) * serve_estimate(0, c.max_batch_edges));
    Ctx *c0 = &S->slot_ctx[0]->c;
    for (; want >= (int64_t(64) << 20); want /= 2) {
      void *p = nullptr;
      if (cudaMallocAsync(&p, size_t(want), c0->stream) == cudaSuccess) {
        cudaFreeAsync(p, c0->stream);
        break;
      }
      cudaGetLastError();
    }
    cudaStreamSynchronize(c0->stream);
  }
  try {
    for (int i = 0; i < c.slots; i++) S->workers.emplace_back(worker, S, i);
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->closing = true;
    }
    S->cv_work.notify_all();
    for (auto &t : S->workers) t.join();
    for (xt_ctx *o : S->slot_ctx) xt_close(o);
    delete srv;
    return XT_ERR_OOM;
  }
  *out = srv;
  return XT_OK;
}

xt_status xt_serve_submit(xt_server *srv, int64_t nv, int64_t ne, const int32_t *src, const int32_t *dst,
                          int64_t *ticket) {
  if (!srv || !ticket || nv < 1 || ne < 0 || (ne > 0 && (!src || !dst))) return XT_ERR_INVALID;
  if (nv > (int64_t(1) << 31) - 1) return XT_ERR_OVERFLOW;
  Server *S = &srv->s;
  Query x;
  x.nv = nv;
  x.ne = ne;
  x.src = src;
  x.dst = dst;
  x.est = serve_estimate(nv, ne);
  x.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->closing) return XT_ERR_CLOSED;
    if (x.est > S->cfg.budget_bytes) {
      S->st.rejected++;
      return XT_ERR_ADMISSION;
    }
    const int64_t t = S->next_ticket++;
    S->q.emplace(t, x);
    S->queue.push_back(t);
    S->st.submitted++;
    S->st.queued = int64_t(S->queue.size());
    *ticket = t;
  }
  S->cv_work.notify_one();
  return XT_OK;
}

// takes the result of a finished query (caller holds the lock)
static xt_status take_result(Server *S, std::unordered_map<int64_t, Query>::iterator it, int64_t *count,
                             double *latency_s) {
  const Query &x = it->second;
  const xt_status s = x.status;
  if (count) *count = x.count;
  if (latency_s) *latency_s = std::chrono::duration<double>(x.t_done - x.t_submit).count();
  S->q.erase(it);
  return s;
}

xt_status xt_serve_poll(xt_server *srv, int64_t ticket, int64_t *count, double *latency_s) {
  if (!srv) return XT_ERR_INVALID;
  Server *S = &srv->s;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->q.find(ticket);
  if (it == S->q.end()) return XT_ERR_INVALID;
  if (it->second.status == XT_ERR_NOT_READY) return XT_ERR_NOT_READY;
  return take_result(S, it, count, latency_s);
}

xt_status xt_serve_wait(xt_server *srv, int64_t ticket, int64_t timeout_ms, int64_t *count, double *latency_s) {
  if (!srv) return XT_ERR_INVALID;
  Server *S = &srv->s;
  std::unique_lock<std::mutex> lk(S->mu);
  auto ready = [&] {
    auto it = S->q.find(ticket);
    return it == S->q.end() || it->second.status != XT_ERR_NOT_READY;
  };
  if (timeout_ms < 0) {
    S->cv_done.wait(lk, ready);
  } else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return XT_ERR_TIMEOUT;
  }
  auto it = S->q.find(ticket);
  if (it == S->q.end()) return XT_ERR_INVALID;
  return take_result(S, it, count, latency_s);
}

xt_status xt_serve_get_stats(xt_server *srv, xt_serve_stats *stats) {
  if (!srv || !stats) return XT_ERR_INVALID;
  Server *S = &srv->s;
  std::lock_guard<std::mutex> lk(S->mu);
  *stats = S->st;
  stats->budget_used = S->budget_used;
  stats->device_peak = S->dev_peak.load();
  stats->queued = int64_t(S->queue.size());
  int64_t l = 0;
  for (xt_ctx *sc : S->slot_ctx) l += sc->c.launches;
  stats->launches = l;
  return XT_OK;
}

int64_t xt_serve_batches(xt_server *srv, xt_serve_batch *out, int64_t max) {
  if (!srv || max < 0 || (max > 0 && !out)) return -1;
  Server *S = &srv->s;
  std::lock_guard<std::mutex> lk(S->mu);
  const int64_t n = std::min<int64_t>(max, int64_t(S->log.size()));
  const size_t first = S->log.size() - size_t(n);
  for (int64_t i = 0; i < n; i++) out[i] = S->log[first + size_t(i)];
  return n;
}

xt_status xt_serve_close(xt_server *srv) {
  if (!srv) return XT_ERR_INVALID;
  Server *S = &srv->s;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->closing = true;
    const Clock::time_point now = Clock::now();
    for (int64_t t : S->queue) {
      Query &x = S->q[t];
      x.status = XT_ERR_CLOSED;
      x.t_done = now;
      S->st.failed++;
    }
    S->queue.clear();
  }
  S->cv_work.notify_all();
  S->cv_done.notify_all();
  for (auto &t : S->workers) t.join();
  for (xt_ctx *sc : S->slot_ctx) xt_close(sc);
  delete srv;
  return XT_OK;
}

}  // extern "C"
