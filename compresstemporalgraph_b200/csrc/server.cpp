// Served form: several resident graphs answer a stream of (algorithm, source, window) queries.
//
// One worker thread per graph takes turns on the device with the others: the graph holding the
// oldest outstanding query goes first, so across graphs the queries are served in arrival order.
// A graph's turn serves the kind of its oldest waiting query together with the other waiting
// queries of that kind that can share its launch, admitted while the device working memory they
// need fits the server's budget (shared by all graphs): BFS queries as one batched traversal
// (tga_bfs_batch), PageRank queries as one strided vector (tga_pagerank_batch_iters, each with its
// own iteration count; fewer than kPrBatchMin of them one call each), CC windows as one
// multi-window seed loop (the CC job, up to 32 windows, run to completion), point queries as one
// launch.  Queries of a kind whose batch costs less than its single calls join the round from
// anywhere in the queue (a batched traversal decodes each list once per level for all its sources);
// the others only from the head of the queue, so they never overtake an earlier query.  A query
// therefore never waits behind work that arrived after it, except for the same-kind queries that
// join its batch, which cost little.  Turns run one at a time: the traversal kernels are
// cooperative launches that occupy every SM, so rounds of different graphs could not overlap on the
// device anyway.  Latency is measured from tga_submit to the moment the result is in the caller's
// buffer.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tga.h"
#include "serve_ops.hpp"

namespace tga {
int fail(int code, const std::string& msg);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  tga_query q;
  int64_t ticket;
  int64_t bytes;
  Clock::time_point submitted;
};

struct Outcome {
  int status = TGA_E_AGAIN;
  double latency_ms = 0.0;
};

struct GraphSlot {
  tga_graph* g = nullptr;
  int32_t nv = 0;
  std::deque<Pending> pending;
  std::thread worker;
  tga_cc_job* cc = nullptr;                 // created at the first CC query
  bool wants_device = false;                // has a round to run (guarded by the server mutex)
  Clock::time_point oldest{};               // submit time of its oldest outstanding query
};

// CC windows per round (the job's capacity).
constexpr int32_t kCcJobWindows = 32;
// PageRank rounds smaller than this run their queries one call each.  The strided batch decodes
// each list once for all its queries but scatters per query, and every query of a batch gets its
// result when the whole batch ends: measured on the 2M/40M graph (windowed, 20 iterations), one
// call per query takes 16.6 ms, a batch of 2 37.2 ms, of 4 46 ms, of 8 73 ms.  From three queries
// the batch costs less device time, but the queries' summed completion times (what latency sees)
// are lower for one call after the other until about eight (4: 184 against 166 ms; 8: 584 against
// 598 ms), so the server batches PageRank only from eight waiting queries.
constexpr size_t kPrBatchMin = 8;

// Device working bytes of one query (per vertex of its graph): BFS arrival + last-enqueued arrival
// + result; PageRank three rank vectors + inverse degree + result; CC the single traversal's arrays.
int64_t query_bytes(const tga_query& q, int32_t nv) {
  if (q.kind == TGA_Q_NEIGHBOR) return 64;
  const int64_t per_vertex = q.kind == TGA_Q_BFS ? 12 : q.kind == TGA_Q_PAGERANK ? 20 : 40;
  return per_vertex * (int64_t)nv;
}

}  // namespace

struct tga_server {
  int64_t budget = 0;
  int64_t in_use = 0;
  std::mutex mu;
  std::condition_variable work_cv, done_cv, turn_cv;
  bool device_busy = false;  // a worker is running its round (one at a time, oldest query first)
  std::vector<std::unique_ptr<GraphSlot>> graphs;
  std::unordered_map<int64_t, Outcome> outcomes;
  int64_t next_ticket = 1;
  bool stopping = false;
  int64_t submitted = 0, completed = 0, failed = 0, rounds = 0, running = 0;
  std::vector<double> latencies;
  bool any_submitted = false;
  Clock::time_point first_submit, last_done;

  void worker(GraphSlot* slot);
  void run_round(GraphSlot* slot, std::vector<Pending>& round);
  void run_cc(GraphSlot* slot, std::vector<Pending>& round);
  void publish(const std::vector<const Pending*>& done, const std::vector<int>& status);
};

// Records the outcome of the queries done[k] (status[k]) and releases their budget.
void tga_server::publish(const std::vector<const Pending*>& done, const std::vector<int>& status) {
  const Clock::time_point now = Clock::now();
  std::lock_guard<std::mutex> lk(mu);
  for (size_t k = 0; k < done.size(); ++k) {
    const Pending& p = *done[k];
    Outcome& o = outcomes[p.ticket];
    o.status = status[k];
    o.latency_ms = std::chrono::duration<double, std::milli>(now - p.submitted).count();
    in_use -= p.bytes;
    if (status[k] == TGA_OK) {
      ++completed;
      latencies.push_back(o.latency_ms);
    } else {
      ++failed;
    }
  }
  running -= (int64_t)done.size();
  last_done = now;
  done_cv.notify_all();
  work_cv.notify_all();
}

void tga_server::run_round(GraphSlot* slot, std::vector<Pending>& round) {
  // BFS: one batched traversal; results published as soon as it is done.
  {
    std::vector<const Pending*> done;
    std::vector<int32_t> src;
    std::vector<int64_t> lo, hi;
    for (const Pending& p : round)
      if (p.q.kind == TGA_Q_BFS) {
        done.push_back(&p);
        src.push_back(p.q.src);
        lo.push_back(p.q.t_lo);
        hi.push_back(p.q.t_hi);
      }
    if (!done.empty()) {
      std::vector<int32_t*> rows(done.size());
      for (size_t k = 0; k < done.size(); ++k) rows[k] = static_cast<int32_t*>(done[k]->q.out);
      const int rc = tga::bfs_batch_rows(slot->g, (int32_t)done.size(), src.data(), lo.data(), hi.data(), rows.data());
      publish(done, std::vector<int>(done.size(), rc));
    }
  }
  // PageRank: one strided batch, each query taken after its own iteration count.
  {
    std::vector<const Pending*> done;
    std::vector<int32_t> iters;
    std::vector<int64_t> lo, hi;
    for (const Pending& p : round)
      if (p.q.kind == TGA_Q_PAGERANK) {
        done.push_back(&p);
        iters.push_back(p.q.iters);  // <= 0: the graph's configured count
        lo.push_back(p.q.t_lo);
        hi.push_back(p.q.t_hi);
      }
    if (!done.empty() && done.size() < kPrBatchMin) {
      for (size_t k = 0; k < done.size(); ++k) {
        const int rc = tga_pagerank(slot->g, iters[k], 0.85f, 0.1f, lo[k], hi[k], static_cast<float*>(done[k]->q.out));
        publish({done[k]}, {rc});
      }
    } else if (!done.empty()) {
      std::vector<float*> rows(done.size());
      for (size_t k = 0; k < done.size(); ++k) rows[k] = static_cast<float*>(done[k]->q.out);
      const int rc = tga::pagerank_batch_rows(slot->g, (int32_t)done.size(), iters.data(), 0.85f, 0.1f, lo.data(),
                                              hi.data(), rows.data());
      publish(done, std::vector<int>(done.size(), rc));
    }
  }
  // Point queries: one launch.
  {
    std::vector<const Pending*> done;
    std::vector<int32_t> x, y;
    std::vector<int64_t> lo, hi;
    for (const Pending& p : round)
      if (p.q.kind == TGA_Q_NEIGHBOR) {
        done.push_back(&p);
        x.push_back(p.q.src);
        y.push_back(p.q.dst);
        lo.push_back(p.q.t_lo);
        hi.push_back(p.q.t_hi);
      }
    if (!done.empty()) {
      std::vector<uint8_t> out(done.size());
      const int rc = tga_is_neighbor(slot->g, (int32_t)done.size(), x.data(), y.data(), lo.data(), hi.data(), out.data());
      for (size_t k = 0; k < done.size(); ++k)
        if (rc == TGA_OK && done[k]->q.out) *static_cast<uint8_t*>(done[k]->q.out) = out[k];
      publish(done, std::vector<int>(done.size(), rc));
    }
  }
  run_cc(slot, round);
}

// CC windows of the round: added to the graph's CC job and run to completion in one step; each
// window's labels go straight to its query's buffer.  A job error fails these windows and drops the
// job (the next CC round makes a new one).
void tga_server::run_cc(GraphSlot* slot, std::vector<Pending>& round) {
  std::vector<const Pending*> cc;
  for (const Pending& p : round)
    if (p.q.kind == TGA_Q_CC) cc.push_back(&p);
  if (cc.empty()) return;
  int rc = TGA_OK;
  if (!slot->cc) rc = tga_cc_job_create(slot->g, kCcJobWindows, TGA_CC_EARLY_EXIT, &slot->cc);
  std::vector<int32_t> slot_of(cc.size(), -1);
  for (size_t k = 0; k < cc.size() && rc == TGA_OK; ++k) rc = tga_cc_job_add(slot->cc, cc[k]->q.t_lo, cc[k]->q.t_hi, &slot_of[k]);
  uint32_t finished = 0;
  if (rc == TGA_OK) rc = tga_cc_job_step(slot->cc, 0.0, &finished);  // budget 0: to completion
  std::vector<int> status(cc.size(), rc);
  if (rc == TGA_OK) {
    for (size_t k = 0; k < cc.size(); ++k)
      status[k] = (finished >> slot_of[k]) & 1u
                      ? tga_cc_job_take(slot->cc, slot_of[k], static_cast<int32_t*>(cc[k]->q.out), nullptr)
                      : TGA_E_CUDA;
  } else {
    if (slot->cc) tga_cc_job_destroy(slot->cc);
    slot->cc = nullptr;
  }
  publish(cc, status);
}

void tga_server::worker(GraphSlot* slot) {
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    work_cv.wait(lk, [&] { return stopping || !slot->pending.empty(); });
    if (slot->pending.empty()) {
      if (stopping) break;
      continue;
    }
    // The kind of the oldest waiting query.  Where one launch for several queries of that kind
    // costs less device time than their single calls (BFS, point queries, PageRank from
    // kPrBatchMin queries on), every waiting query of the kind joins the round, though some arrived
    // after queries of other kinds; otherwise (CC windows, which gain nothing from sharing a launch,
    // and fewer PageRank queries) only the queries of the kind at the head of the queue, so none
    // overtakes an earlier query.  Admitted while they fit the budget (at least one when nothing
    // else runs); CC at most a job's windows.
    const int32_t kind = slot->pending.front().q.kind;
    size_t waiting = 0;
    for (const Pending& p : slot->pending) waiting += p.q.kind == kind;
    const bool gather = kind == TGA_Q_BFS || kind == TGA_Q_NEIGHBOR || (kind == TGA_Q_PAGERANK && waiting >= kPrBatchMin);
    std::vector<Pending> round;
    std::deque<Pending> rest;
    bool full = false, head = true;
    while (!slot->pending.empty()) {
      Pending p = slot->pending.front();
      slot->pending.pop_front();
      head = head && p.q.kind == kind;
      if (full || p.q.kind != kind || (!gather && !head) || (kind == TGA_Q_CC && (int32_t)round.size() >= kCcJobWindows) ||
          (in_use + p.bytes > budget && !(round.empty() && in_use == 0))) {
        if (p.q.kind == kind && !round.empty()) full = full || in_use + p.bytes > budget;
        rest.push_back(p);
        continue;
      }
      in_use += p.bytes;
      round.push_back(p);
    }
    slot->pending.swap(rest);
    if (round.empty()) {  // the budget is held by other graphs: wait until some is released
      work_cv.wait(lk);
      continue;
    }
    // Device turn: the graph holding the oldest outstanding query first.
    Clock::time_point oldest = Clock::time_point::max();
    for (const Pending& p : round) oldest = std::min(oldest, p.submitted);
    for (const Pending& p : slot->pending) oldest = std::min(oldest, p.submitted);
    slot->oldest = oldest;
    slot->wants_device = true;
    turn_cv.wait(lk, [&] {
      if (device_busy) return false;
      for (const auto& o : graphs)
        if (o.get() != slot && o->wants_device && o->oldest < slot->oldest) return false;
      return true;
    });
    device_busy = true;
    slot->wants_device = false;
    ++rounds;
    running += (int64_t)round.size();
    lk.unlock();
    run_round(slot, round);
    lk.lock();
    device_busy = false;
    turn_cv.notify_all();
  }
  lk.unlock();
  if (slot->cc) tga_cc_job_destroy(slot->cc);
  slot->cc = nullptr;
}

using tga::fail;

extern "C" {

int tga_server_create(int64_t budget_bytes, tga_server** out) {
  if (!out || budget_bytes <= 0) return fail(TGA_E_ARG, "tga_server_create: need a positive budget and an output");
  *out = new tga_server();
  (*out)->budget = budget_bytes;
  return TGA_OK;
}

int tga_server_add_graph(tga_server* s, tga_graph* g, int32_t* graph_id) {
  if (!s || !g) return fail(TGA_E_ARG, "null server or graph");
  tga_info info;
  if (int rc = tga_get_info(g, &info)) return rc;
  auto slot = std::make_unique<GraphSlot>();
  slot->g = g;
  slot->nv = info.max_vertex;
  std::lock_guard<std::mutex> lk(s->mu);
  const int32_t id = (int32_t)s->graphs.size();
  GraphSlot* raw = slot.get();
  s->graphs.push_back(std::move(slot));
  raw->worker = std::thread([s, raw] { s->worker(raw); });
  if (graph_id) *graph_id = id;
  return TGA_OK;
}

int tga_submit(tga_server* s, const tga_query* q, int64_t* ticket) {
  if (!s || !q) return fail(TGA_E_ARG, "null server or query");
  if (q->kind < TGA_Q_BFS || q->kind > TGA_Q_NEIGHBOR) return fail(TGA_E_ARG, "unknown query kind");
  if (q->kind == TGA_Q_NEIGHBOR ? q->t_lo > q->t_hi : q->t_lo >= q->t_hi) return fail(TGA_E_ARG, "empty time window");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return fail(TGA_E_ARG, "server is stopping");
  if (q->graph < 0 || q->graph >= (int32_t)s->graphs.size()) return fail(TGA_E_ARG, "unknown graph id");
  GraphSlot* slot = s->graphs[(size_t)q->graph].get();
  if (q->kind == TGA_Q_BFS && (q->src < 0 || q->src >= slot->nv)) return fail(TGA_E_ARG, "source out of range");
  Pending p{*q, s->next_ticket++, query_bytes(*q, slot->nv), Clock::now()};
  if (p.bytes > s->budget) return fail(TGA_E_OOM, "query needs more device memory than the server's budget");
  if (!s->any_submitted) {
    s->any_submitted = true;
    s->first_submit = p.submitted;
  }
  s->outcomes[p.ticket] = Outcome{};
  slot->pending.push_back(p);
  ++s->submitted;
  if (ticket) *ticket = p.ticket;
  s->work_cv.notify_all();
  return TGA_OK;
}

int tga_poll(tga_server* s, int64_t ticket, double* latency_ms) {
  if (!s) return fail(TGA_E_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->outcomes.find(ticket);
  if (it == s->outcomes.end()) return fail(TGA_E_ARG, "unknown ticket");
  if (latency_ms) *latency_ms = it->second.latency_ms;
  return it->second.status;
}

int tga_server_drain(tga_server* s) {
  if (!s) return fail(TGA_E_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  s->done_cv.wait(lk, [&] { return s->completed + s->failed == s->submitted; });
  return TGA_OK;
}

int tga_server_get_stats(tga_server* s, tga_server_stats* out) {
  if (!s || !out) return fail(TGA_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof *out);
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->rounds = s->rounds;
  if (!s->latencies.empty()) {
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l[(size_t)std::min<double>((double)l.size() - 1, p * (double)(l.size() - 1) + 0.5)]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    out->mean_ms = sum / (double)l.size();
    const double span = std::chrono::duration<double>(s->last_done - s->first_submit).count();
    out->queries_per_s = span > 0 ? (double)s->completed / span : 0.0;
  }
  return TGA_OK;
}

int tga_server_destroy(tga_server* s) {
  if (!s) return fail(TGA_E_ARG, "null server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->work_cv.notify_all();
  }
  for (auto& g : s->graphs)
    if (g->worker.joinable()) g->worker.join();
  delete s;
  return TGA_OK;
}

}  // extern "C"
