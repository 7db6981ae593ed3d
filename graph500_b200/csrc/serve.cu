// Serving loop: several graphs resident on one device, BFS queries admitted
// as they arrive and batched into multi-source launches (g500_msbfs), with
// p50/p99 latency reported beside throughput.  No counterpart in the
// reference, whose driver runs one root at a time (main.cc:105-160); each
// query's levels equal that root's (pred >> 48) from run_bfs (bfs.hpp:1203,
// :2470).
//
// One engine thread owns every device handle.  Per graph it keeps up to
// max_workers_per_graph multi-source handles ("workers", each with its own
// stream and workspace).  A worker is created only when a query of its graph
// is waiting, every existing worker of the graph is busy, and the device
// still has the workspace plus hbm_reserve_bytes free (admission by free HBM).
// An idle worker takes up to max_batch waiting queries of its graph at once
// (lane width 32/64/128, the smallest that holds them) and launches them
// asynchronously; queries that arrive meanwhile wait for the next free
// worker, so batches form from whatever arrived while the device was busy
// (continuous batching).  Graphs are served oldest waiting query first, and
// a graph whose launch does not fit in the free blocks reserves them, so that
// small launches of other graphs cannot starve a large graph (without that,
// 4 graphs of SCALE 18-24 served only 21k of 30k q/s offered, p99 0.3 s; with
// it 29.7k, p99 12 ms).  Optionally (batch_target > 0) a second launch of a
// graph waits until that many of its queries wait; off by default, since it
// measured worse at 30k q/s (p99 17-62 ms).  Launches of different workers
// run concurrently on
// their own streams; the sum of their persistent-kernel grids never exceeds
// the device's co-resident blocks, so every grid barrier can complete.
#include "g500_internal.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace {

using clk = std::chrono::steady_clock;

struct Query {
  int64_t id = 0;
  uint64_t tag = 0;
  int graph = 0;
  int64_t root = 0;
  uint8_t* levels_out = nullptr;
  int slot = -1;          // delivery slot of a load-generator query (g500_server_set_delivery)
  bool internal = false;  // submitted by the load generator: kept out of poll
  g500_query_result res{};
};

struct Worker {
  g500_msbfs* ms = nullptr;
  int graph = -1;
  bool busy = false;
  int blocks = 0;
  int lanes = 0;
  double t_start_us = 0;
  std::vector<int64_t> qids;
};

// A plain BFS handle that serves one query at a time, for graphs whose queue
// is short: a one-root multi-source launch costs far more than one BFS.
struct PlainWorker {
  g500_bfs* bfs = nullptr;
  bool busy = false;
  int units = 0;  // share of the block budget (in 256-thread blocks)
  double t_start_us = 0;
  int64_t qid = -1;
};

uint64_t splitmix64(uint64_t* x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double unit_double(uint64_t* x) { return (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

struct g500_server {
  std::vector<g500_graph*> graphs;
  g500_server_config cfg{};
  int device = 0;
  clk::time_point t0;

  std::mutex mu;
  std::condition_variable cv_work;  // engine: new queries or stop
  std::condition_variable cv_done;  // callers: queries completed
  std::unordered_map<int64_t, Query> queries;
  std::vector<std::deque<int64_t>> pending;  // batched mode: per graph
  std::deque<int64_t> fifo;                  // plain mode: arrival order
  std::deque<int64_t> completed;             // ids ready for poll
  int64_t next_id = 0, finished = 0;
  bool stop = false;
  int engine_status = G500_OK;
  std::string engine_error;

  // engine thread only
  std::vector<std::vector<Worker>> workers;
  std::vector<std::vector<PlainWorker>> pworkers;  // per graph
  std::vector<int> plain_below;    // queues up to this long go to plain BFS runs
  std::vector<int> pblocks;        // grid of a graph's plain runs (512-thread blocks)
  std::vector<uint64_t> pws_bytes; // workspace of one plain handle
  std::vector<int> blocks;         // grid of each graph's launches
  std::vector<double> alpha;
  std::vector<uint64_t> ws_bytes;  // workspace of one worker
  std::vector<char> no_more;       // the last worker creation failed for lack of memory
  int capacity = 0, inflight_blocks = 0;
  std::vector<g500_bfs*> plain;    // plain mode: one handle per graph
  int64_t* d_pred = nullptr;
  int64_t* h_pred = nullptr;
  int64_t pred_cap = 0;

  // result delivery of load-generator queries: per graph a ring of level
  // buffers (device or pinned host memory), one per query in flight
  int delivery = G500_DELIVER_NONE;
  std::vector<std::vector<uint8_t*>> slots;   // per graph
  std::vector<std::vector<int>> free_slots;   // per graph (engine thread)

  std::atomic<int64_t> launches{0}, lanes_used{0};
  std::atomic<int> in_flight{0}, max_in_flight{0}, nworkers{0};
  std::thread engine;

  double now_us() const { return std::chrono::duration<double, std::micro>(clk::now() - t0).count(); }
};

namespace {

void fail_engine(g500_server* s, int st) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->engine_status == G500_OK) {
    s->engine_status = st;
    s->engine_error = g500_last_error();
  }
}

// Record the results of finished queries and wake the callers.
void finish_queries(g500_server* s, const std::vector<int64_t>& qids, int status, const int64_t* reached,
                    const int64_t* nedge, double start_us, int batch, int lanes) {
  const double done = s->now_us();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t i = 0; i < qids.size(); ++i) {
      auto it = s->queries.find(qids[i]);
      if (it == s->queries.end()) continue;
      g500_query_result& r = it->second.res;
      r.status = status;
      r.reached = reached ? reached[i] : 0;
      r.nedge = nedge ? nedge[i] : 0;
      r.start_us = start_us;
      r.done_us = done;
      r.batch_size = batch;
      r.lane_width = lanes;
      if (it->second.slot >= 0) {
        s->free_slots[(size_t)it->second.graph].push_back(it->second.slot);
        it->second.slot = -1;
        it->second.levels_out = nullptr;
      }
      if (!it->second.internal) s->completed.push_back(qids[i]);
      ++s->finished;
    }
  }
  s->cv_done.notify_all();
}

int new_worker(g500_server* s, int g, Worker* out) {
  size_t free_b = 0, total_b = 0;
  G500_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if ((uint64_t)free_b < s->ws_bytes[(size_t)g] + s->cfg.hbm_reserve_bytes)
    return g500::set_error(G500_E_NOMEM, "no room for another worker on graph %d", g);
  Worker w;
  w.graph = g;
  G500_TRY(g500_msbfs_create(s->graphs[(size_t)g], &w.ms));
  int st = g500_msbfs_set_params(w.ms, 64, s->alpha[(size_t)g], 1);
  if (st == G500_OK) st = g500_msbfs_set_root_stats(w.ms, 1);
  if (st == G500_OK) st = g500_msbfs_set_grid(w.ms, s->blocks[(size_t)g]);
  if (st != G500_OK) {
    g500_msbfs_destroy(w.ms);
    return st;
  }
  w.blocks = s->blocks[(size_t)g];
  *out = std::move(w);
  s->nworkers.fetch_add(1);
  return G500_OK;
}

// Poll the busy workers; returns whether any finished.
bool reap(g500_server* s) {
  bool any = false;
  for (auto& ps : s->pworkers)
    for (PlainWorker& w : ps) {
      if (!w.busy) continue;
      int done = 0;
      int st = g500::bfs_poll(w.bfs, &done);
      if (st == G500_OK && !done) continue;
      int64_t reached = 0, nedge = 0;
      const int st2 = g500::bfs_complete(w.bfs, &reached, &nedge);
      if (st == G500_OK) st = st2;
      const std::vector<int64_t> ids{w.qid};
      finish_queries(s, ids, st, &reached, &nedge, w.t_start_us, 1, 0);
      w.busy = false;
      w.qid = -1;
      s->inflight_blocks -= w.units;
      s->in_flight.fetch_sub(1);
      any = true;
    }
  for (auto& ws : s->workers)
    for (Worker& w : ws) {
      if (!w.busy) continue;
      int done = 0;
      int st = g500_msbfs_poll(w.ms, &done);
      if (st == G500_OK && !done) continue;
      g500_msbfs_stats ms{};
      if (st == G500_OK) st = g500_msbfs_wait(w.ms, &ms);
      else g500_msbfs_wait(w.ms, nullptr);  // the poll failed: retire the launch all the same
      std::vector<int64_t> reached(w.qids.size(), 0), nedge(w.qids.size(), 0);
      if (st == G500_OK) st = g500_msbfs_root_stats(w.ms, reached.data(), nedge.data());
      finish_queries(s, w.qids, st, reached.data(), nedge.data(), w.t_start_us, (int)w.qids.size(), w.lanes);
      w.busy = false;
      w.qids.clear();
      s->inflight_blocks -= w.blocks;
      s->in_flight.fetch_sub(1);
      any = true;
    }
  return any;
}

void free_delivery(g500_server* s) {
  for (auto& gs : s->slots)
    for (uint8_t* p : gs) {
      if (s->delivery == G500_DELIVER_HOST) cudaFreeHost(p);
      else cudaFree(p);
    }
  s->slots.clear();
  s->free_slots.clear();
  s->delivery = G500_DELIVER_NONE;
}

// A load-generator query with delivery on gets a free level buffer of its
// graph as its destination (caller holds s->mu); false when none is free.
bool take_slot(g500_server* s, int g, Query* q) {
  if (s->delivery == G500_DELIVER_NONE || !q->internal || q->levels_out) return true;
  auto& fs = s->free_slots[(size_t)g];
  if (fs.empty()) return false;
  q->slot = fs.back();
  fs.pop_back();
  q->levels_out = s->slots[(size_t)g][(size_t)q->slot];
  return true;
}

// Launch the waiting queries of every graph that has an idle (or admissible
// new) worker and room in the block budget.  Graphs are served oldest
// waiting query first.  A graph whose launch does
// not fit in the free blocks reserves them: graphs behind it may only start
// launches that leave its share free, so that a large graph's launch is not
// starved by a stream of small launches of other graphs.
bool dispatch(g500_server* s) {
  bool any = false;
  const int ng = (int)s->graphs.size();
  std::vector<std::pair<double, int>> order;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int g = 0; g < ng; ++g)
      if (!s->pending[(size_t)g].empty())
        order.emplace_back(s->queries[s->pending[(size_t)g].front()].res.arrival_us, g);
  }
  std::sort(order.begin(), order.end());
  int reserved = 0;  // blocks kept free for older graphs that could not start
  for (const auto& og : order) {
    const int g = og.second;
    for (;;) {
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->pending[(size_t)g].empty()) break;
      }
      size_t waiting;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        waiting = s->pending[(size_t)g].size();
      }
      if ((int)waiting <= s->plain_below[(size_t)g] && !s->pworkers[(size_t)g].empty()) {
        // a short queue: one plain BFS per query
        PlainWorker* pw = nullptr;
        for (PlainWorker& x : s->pworkers[(size_t)g])
          if (!x.busy) {
            pw = &x;
            break;
          }
        if (pw && s->inflight_blocks + pw->units + reserved > s->capacity) {
          reserved += pw->units;
          break;
        }
        if (pw) {
          int64_t id;
          int64_t root;
          uint8_t* dst;
          {
            std::lock_guard<std::mutex> lk(s->mu);
            id = s->pending[(size_t)g].front();
            Query& q = s->queries[id];
            if (!take_slot(s, g, &q)) break;  // every delivery slot is in use: wait for one
            s->pending[(size_t)g].pop_front();
            root = q.root;
            dst = q.levels_out;
          }
          pw->t_start_us = s->now_us();
          const int st = g500::bfs_launch_levels(pw->bfs, root, dst);
          if (st != G500_OK) {
            const std::vector<int64_t> ids{id};
            finish_queries(s, ids, st, nullptr, nullptr, pw->t_start_us, 1, 0);
            continue;
          }
          pw->busy = true;
          pw->qid = id;
          s->inflight_blocks += pw->units;
          s->launches.fetch_add(1);
          s->lanes_used.fetch_add(1);
          const int f = s->in_flight.fetch_add(1) + 1;
          int m = s->max_in_flight.load();
          while (f > m && !s->max_in_flight.compare_exchange_weak(m, f)) {
          }
          any = true;
          continue;
        }
        break;  // the plain worker is busy or the budget is full: wait for it
      }
      if (s->inflight_blocks + s->blocks[(size_t)g] + reserved > s->capacity) {
        reserved += s->blocks[(size_t)g];
        break;
      }
      // hold a second launch of this graph until it fills batch_target lanes
      if (s->cfg.batch_target > 0 && (int)waiting < s->cfg.batch_target) {
        bool running = false;
        for (const Worker& x : s->workers[(size_t)g]) running |= x.busy;
        if (running) break;
      }
      Worker* w = nullptr;
      for (Worker& x : s->workers[(size_t)g])
        if (!x.busy) {
          w = &x;
          break;
        }
      if (!w) {
        if ((int)s->workers[(size_t)g].size() >= s->cfg.max_workers_per_graph || s->no_more[(size_t)g]) break;
        Worker nw;
        const int st = new_worker(s, g, &nw);
        if (st == G500_E_NOMEM) {
          s->no_more[(size_t)g] = 1;
          if (s->workers[(size_t)g].empty()) fail_engine(s, st);
          break;
        }
        if (st != G500_OK) {
          fail_engine(s, st);
          return any;
        }
        s->workers[(size_t)g].push_back(std::move(nw));
        w = &s->workers[(size_t)g].back();
      }
      std::vector<int64_t> roots;
      std::vector<uint8_t*> dsts;
      w->qids.clear();
      {
        std::lock_guard<std::mutex> lk(s->mu);
        auto& pq = s->pending[(size_t)g];
        while (!pq.empty() && (int)w->qids.size() < s->cfg.max_batch) {
          const int64_t id = pq.front();
          Query& q = s->queries[id];
          if (!take_slot(s, g, &q)) break;
          pq.pop_front();
          w->qids.push_back(id);
          roots.push_back(q.root);
          dsts.push_back(q.levels_out);
        }
      }
      const int n = (int)roots.size();
      if (n == 0) break;  // every delivery slot is in use
      const int lanes = n <= 32 ? 32 : (n <= 64 ? 64 : 128);
      int st = g500_msbfs_set_params(w->ms, lanes, s->alpha[(size_t)g], 1);
      w->t_start_us = s->now_us();
      if (st == G500_OK) st = g500::msbfs_launch_to(w->ms, roots.data(), n, dsts.data());
      if (st != G500_OK) {
        finish_queries(s, w->qids, st, nullptr, nullptr, w->t_start_us, n, lanes);
        w->qids.clear();
        continue;
      }
      w->busy = true;
      w->lanes = lanes;
      s->inflight_blocks += w->blocks;
      s->launches.fetch_add(1);
      s->lanes_used.fetch_add(n);
      const int f = s->in_flight.fetch_add(1) + 1;
      int m = s->max_in_flight.load();
      while (f > m && !s->max_in_flight.compare_exchange_weak(m, f)) {
      }
      any = true;
    }
  }
  return any;
}

// Plain mode: one query at a time through g500_bfs_run.
bool run_plain_one(g500_server* s) {
  int64_t id;
  int g;
  int64_t root;
  uint8_t* dst;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fifo.empty()) return false;
    id = s->fifo.front();
    s->fifo.pop_front();
    const Query& q = s->queries[id];
    g = q.graph;
    root = q.root;
    dst = q.levels_out;
  }
  const double t = s->now_us();
  s->in_flight.fetch_add(1);
  int m = s->max_in_flight.load();
  while (1 > m && !s->max_in_flight.compare_exchange_weak(m, 1)) {
  }
  g500_bfs_stats st{};
  int rc = g500_bfs_run(s->plain[(size_t)g], root, s->d_pred, 1, &st);
  const int64_t nolv = s->graphs[(size_t)g]->nolv;
  if (rc == G500_OK && dst) {
    cudaError_t e = cudaMemcpy(s->h_pred, s->d_pred, sizeof(int64_t) * (size_t)nolv, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = g500::cuda_error(e, "pred copy", __FILE__, __LINE__);
    for (int64_t v = 0; rc == G500_OK && v < nolv; ++v) {
      const int64_t p = s->h_pred[v];
      dst[v] = p == -1 ? (uint8_t)255 : (uint8_t)std::min<int64_t>((p >> 48) & 0xFFFF, 255);
    }
  }
  s->launches.fetch_add(1);
  s->lanes_used.fetch_add(1);
  s->in_flight.fetch_sub(1);
  const std::vector<int64_t> ids{id};
  finish_queries(s, ids, rc, &st.reached, &st.nedge, t, 1, 1);
  return true;
}

void engine_main(g500_server* s) {
  cudaSetDevice(s->device);
  const bool plain = s->cfg.mode == G500_SERVE_PLAIN;
  for (;;) {
    bool progress = plain ? run_plain_one(s) : reap(s);
    if (!plain) progress |= dispatch(s);
    if (progress) continue;
    std::unique_lock<std::mutex> lk(s->mu);
    bool waiting = !s->fifo.empty();
    for (auto& pq : s->pending) waiting |= !pq.empty();
    if (s->stop && !waiting && s->in_flight.load() == 0) break;
    if (s->in_flight.load() > 0) {
      // launches in flight: come back soon to collect them
      s->cv_work.wait_for(lk, std::chrono::microseconds(20));
    } else if (!waiting || s->engine_status != G500_OK) {
      s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
    } else {
      // queries wait but nothing can start (no worker admitted): retry shortly
      s->cv_work.wait_for(lk, std::chrono::microseconds(200));
    }
  }
}

int submit_at(g500_server* s, int graph, int64_t root, uint64_t tag, uint8_t* levels_out, double arrival_us,
              bool internal, int64_t* id_out) {
  if (graph < 0 || graph >= (int)s->graphs.size())
    return g500::set_error(G500_E_INVAL, "graph %d outside [0, %d)", graph, (int)s->graphs.size());
  const g500_graph* g = s->graphs[(size_t)graph];
  if (root < 0 || root >= g->nolv)
    return g500::set_error(G500_E_INVAL, "root %lld outside [0, %lld)", (long long)root, (long long)g->nolv);
  int64_t id;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return g500::set_error(G500_E_STATE, "server is stopping");
    if (s->engine_status != G500_OK)
      return g500::set_error(s->engine_status, "server engine failed: %s", s->engine_error.c_str());
    id = s->next_id++;
    Query q;
    q.id = id;
    q.tag = tag;
    q.graph = graph;
    q.root = root;
    q.levels_out = levels_out;
    q.internal = internal;
    q.res.id = id;
    q.res.tag = tag;
    q.res.graph = graph;
    q.res.root = root;
    q.res.arrival_us = arrival_us;
    s->queries.emplace(id, q);
    if (s->cfg.mode == G500_SERVE_PLAIN) s->fifo.push_back(id);
    else s->pending[(size_t)graph].push_back(id);
  }
  s->cv_work.notify_one();
  if (id_out) *id_out = id;
  return G500_OK;
}

// plain_below for graph g: the given value, or (negative) the number of
// queries whose one-at-a-time plain runs cost what one multi-source launch of
// a single root costs, both timed here on a few roots (at most 32).
int calibrate_plain(g500_server* s, int g, int given) {
  if (given >= 0) {
    s->plain_below[(size_t)g] = given;
    return G500_OK;
  }
  g500_graph* gr = s->graphs[(size_t)g];
  int64_t roots[4];
  int found = 0;
  G500_TRY(g500_graph_find_roots(gr, 4, 2, 3, roots, &found));
  if (found == 0) return G500_OK;
  g500_bfs* b = s->pworkers[(size_t)g][0].bfs;
  g500_msbfs* m = s->workers[(size_t)g][0].ms;
  G500_TRY(g500_msbfs_set_params(m, 32, s->alpha[(size_t)g], 1));
  double tp = 1e300, tm = 1e300;
  for (int rep = 0; rep < 3; ++rep)
    for (int i = 0; i < found; ++i) {
      const auto t0 = clk::now();
      G500_TRY(g500::bfs_launch_levels(b, roots[i], nullptr));
      G500_TRY(g500::bfs_complete(b, nullptr, nullptr));
      tp = std::min(tp, std::chrono::duration<double>(clk::now() - t0).count());
      g500_msbfs_stats st;
      const auto t1 = clk::now();
      G500_TRY(g500_msbfs_run(m, &roots[i], 1, nullptr, 0, &st));
      tm = std::min(tm, std::chrono::duration<double>(clk::now() - t1).count());
    }
  s->plain_below[(size_t)g] = (int)std::max(0.0, std::min(32.0, std::floor(tm / tp)));
  return G500_OK;
}

}  // namespace

extern "C" int g500_server_default_config(g500_server_config* cfg) {
  if (!cfg) return g500::set_error(G500_E_INVAL, "null argument");
  memset(cfg, 0, sizeof(*cfg));
  cfg->max_batch = 128;
  cfg->max_workers_per_graph = 2;
  cfg->mode = G500_SERVE_BATCHED;
  cfg->vertices_per_block = 4096;
  cfg->hbm_reserve_bytes = 1ull << 30;
  cfg->alpha = 6.0;
  cfg->max_grid_fraction = 0.5;
  cfg->plain_below = -1;
  cfg->batch_target = 0;
  return G500_OK;
}

extern "C" int g500_server_create(g500_graph* const* graphs, int num_graphs, const g500_server_config* cfg,
                                  g500_server** out) {
  if (!graphs || num_graphs < 1 || !out) return g500::set_error(G500_E_INVAL, "bad argument");
  g500_server_config c;
  g500_server_default_config(&c);
  if (cfg) c = *cfg;
  if (c.max_batch < 1 || c.max_batch > 128) return g500::set_error(G500_E_INVAL, "max_batch %d not in 1..128", c.max_batch);
  if (c.max_workers_per_graph < 1) return g500::set_error(G500_E_INVAL, "max_workers_per_graph must be >= 1");
  if (c.mode != G500_SERVE_BATCHED && c.mode != G500_SERVE_PLAIN) return g500::set_error(G500_E_INVAL, "unknown mode");
  if (c.vertices_per_block < 1) c.vertices_per_block = 4096;
  if (!(c.alpha > 0)) c.alpha = 6.0;
  if (!(c.max_grid_fraction > 0) || c.max_grid_fraction > 1) c.max_grid_fraction = 1.0;
  for (int i = 0; i < num_graphs; ++i) {
    if (!graphs[i]) return g500::set_error(G500_E_INVAL, "graph %d is null", i);
    if (graphs[i]->device != graphs[0]->device) return g500::set_error(G500_E_INVAL, "graphs on different devices");
  }
  g500_server* s = new g500_server();
  s->graphs.assign(graphs, graphs + num_graphs);
  s->cfg = c;
  s->device = graphs[0]->device;
  s->t0 = clk::now();
  s->pending.resize((size_t)num_graphs);
  s->workers.resize((size_t)num_graphs);
  s->pworkers.resize((size_t)num_graphs);
  s->plain_below.assign((size_t)num_graphs, 0);
  s->pblocks.assign((size_t)num_graphs, 0);
  s->blocks.assign((size_t)num_graphs, 0);
  s->alpha.assign((size_t)num_graphs, c.alpha);
  s->ws_bytes.assign((size_t)num_graphs, 0);
  s->no_more.assign((size_t)num_graphs, 0);
  int st = G500_OK;
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) st = g500::cuda_error(e, "cudaSetDevice", __FILE__, __LINE__);
  if (c.mode == G500_SERVE_BATCHED) {
    // one worker per graph up front: it fixes the grid sizes and the block budget
    for (int g = 0; g < num_graphs && st == G500_OK; ++g) {
      st = g500_msbfs_workspace_bytes(graphs[g], &s->ws_bytes[(size_t)g]);
      Worker w;
      if (st == G500_OK) st = g500_msbfs_create(graphs[g], &w.ms);
      int full = 0;
      if (st == G500_OK) st = g500_msbfs_get_grid(w.ms, 64, nullptr, &full);
      if (st == G500_OK) {
        s->capacity = s->capacity == 0 ? full : std::min(s->capacity, full);
        const int64_t want = (graphs[g]->nlv + c.vertices_per_block - 1) / c.vertices_per_block;
        const int64_t cap = std::max<int64_t>(1, (int64_t)(c.max_grid_fraction * full));
        s->blocks[(size_t)g] = (int)std::max<int64_t>(std::min<int64_t>(want, cap), std::min<int64_t>(16, cap));
        st = g500_msbfs_set_params(w.ms, 64, c.alpha, 1);
      }
      if (st == G500_OK) st = g500_msbfs_set_root_stats(w.ms, 1);
      if (st == G500_OK) st = g500_msbfs_set_grid(w.ms, s->blocks[(size_t)g]);
      if (w.ms) {
        w.graph = g;
        w.blocks = s->blocks[(size_t)g];
        s->workers[(size_t)g].push_back(std::move(w));
        s->nworkers.fetch_add(1);
      }
      // one plain handle per graph, on the same share of the device
      if (st == G500_OK && c.plain_below != 0) {
        PlainWorker pw;
        st = g500_bfs_create(graphs[g], &pw.bfs);
        if (st == G500_OK) {
          const int pb = std::max(1, s->blocks[(size_t)g] / 2);  // 512-thread blocks
          st = g500_bfs_set_grid(pw.bfs, pb);
          pw.units = 2 * pb;
          s->pblocks[(size_t)g] = pb;
        }
        if (pw.bfs) s->pworkers[(size_t)g].push_back(pw);
        if (st == G500_OK) st = calibrate_plain(s, g, c.plain_below);
      }
    }
  } else {
    s->plain.assign((size_t)num_graphs, nullptr);
    for (int g = 0; g < num_graphs && st == G500_OK; ++g) {
      st = g500_bfs_create(graphs[g], &s->plain[(size_t)g]);
      s->pred_cap = std::max<int64_t>(s->pred_cap, graphs[g]->nolv);
    }
    if (st == G500_OK) {
      e = cudaMalloc(&s->d_pred, sizeof(int64_t) * (size_t)s->pred_cap);
      if (e == cudaSuccess) e = cudaHostAlloc(&s->h_pred, sizeof(int64_t) * (size_t)s->pred_cap, cudaHostAllocDefault);
      if (e != cudaSuccess) st = g500::cuda_error(e, "plain-mode buffers", __FILE__, __LINE__);
    }
  }
  // The other workers are created now, round robin over the graphs, as many
  // as free HBM admits: creating one inside the loop allocates and builds its
  // hub tables on a busy device, which held every waiting query for 0.1-0.5 s.
  if (st == G500_OK && c.mode == G500_SERVE_BATCHED)
    for (int k = 1; k < c.max_workers_per_graph && st == G500_OK; ++k)
      for (int g = 0; g < num_graphs && st == G500_OK; ++g) {
        if (s->no_more[(size_t)g]) continue;
        Worker nw;
        const int ws = new_worker(s, g, &nw);
        if (ws == G500_E_NOMEM) s->no_more[(size_t)g] = 1;
        else if (ws != G500_OK) st = ws;
        else s->workers[(size_t)g].push_back(std::move(nw));
      }
  if (st != G500_OK) {
    g500_server_destroy(s);
    return st;
  }
  s->engine = std::thread(engine_main, s);
  *out = s;
  return G500_OK;
}

extern "C" int g500_server_submit(g500_server* s, int graph, int64_t root, uint64_t tag, uint8_t* levels_out,
                                  int64_t* id) {
  if (!s) return g500::set_error(G500_E_INVAL, "null handle");
  return submit_at(s, graph, root, tag, levels_out, s->now_us(), false, id);
}

extern "C" int g500_server_poll(g500_server* s, g500_query_result* out, int max_results, int* num, int wait_us) {
  if (!s || !out || !num || max_results < 1) return g500::set_error(G500_E_INVAL, "bad argument");
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->completed.empty() && wait_us > 0)
    s->cv_done.wait_for(lk, std::chrono::microseconds(wait_us), [&] { return !s->completed.empty(); });
  int n = 0;
  while (n < max_results && !s->completed.empty()) {
    const int64_t id = s->completed.front();
    s->completed.pop_front();
    auto it = s->queries.find(id);
    if (it == s->queries.end()) continue;
    out[n++] = it->second.res;
    s->queries.erase(it);
  }
  *num = n;
  return G500_OK;
}

extern "C" int g500_server_drain(g500_server* s, int timeout_ms) {
  if (!s) return g500::set_error(G500_E_INVAL, "null handle");
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms > 0 ? timeout_ms : 60000), [&] {
    return s->finished == s->next_id || s->engine_status != G500_OK;
  });
  if (s->engine_status != G500_OK)
    return g500::set_error(s->engine_status, "server engine failed: %s", s->engine_error.c_str());
  if (!ok) return g500::set_error(G500_E_TIMEOUT, "queries still running after %d ms", timeout_ms);
  return G500_OK;
}

extern "C" int g500_server_info(g500_server* s, g500_server_info_t* info) {
  if (!s || !info) return g500::set_error(G500_E_INVAL, "null argument");
  memset(info, 0, sizeof(*info));
  info->launches = s->launches.load();
  info->queries_launched = s->lanes_used.load();
  info->workers = s->nworkers.load();
  info->max_in_flight = s->max_in_flight.load();
  info->block_capacity = s->capacity;
  std::lock_guard<std::mutex> lk(s->mu);
  info->submitted = s->next_id;
  info->finished = s->finished;
  return G500_OK;
}

extern "C" int g500_server_run_poisson(g500_server* s, double rate_qps, int64_t num_queries, uint64_t seed,
                                       int64_t warmup, g500_serve_report* rep) {
  if (!s || !rep || !(rate_qps > 0) || num_queries < 1 || warmup < 0 || warmup >= num_queries)
    return g500::set_error(G500_E_INVAL, "bad argument");
  const int ng = (int)s->graphs.size();
  // the arrival schedule, graphs and roots first (seeded), so that the
  // stream does not depend on timing
  uint64_t x = seed;
  std::vector<double> at((size_t)num_queries);
  std::vector<int> gs((size_t)num_queries);
  std::vector<int64_t> rs((size_t)num_queries);
  double t = s->now_us() + 1000.0;
  for (int64_t k = 0; k < num_queries; ++k) {
    t += -std::log(1.0 - unit_double(&x)) / rate_qps * 1e6;
    at[(size_t)k] = t;
    const int g = std::min(ng - 1, (int)(unit_double(&x) * ng));
    gs[(size_t)k] = g;
    const g500_graph* gr = s->graphs[(size_t)g];
    int64_t v;
    for (int tries = 0;; ++tries) {  // uniform over vertices with at least one edge
      v = std::min<int64_t>(gr->nolv - 1, (int64_t)(unit_double(&x) * (double)gr->nolv));
      if ((gr->h_has_edge_orig[(size_t)(v >> 5)] >> (v & 31)) & 1u) break;
      if (tries > 1000000) return g500::set_error(G500_E_INVAL, "graph %d has no vertex with edges", g);
    }
    rs[(size_t)k] = v;
  }
  const int64_t l0 = s->launches.load(), q0 = s->lanes_used.load();
  s->max_in_flight.store(0);
  std::vector<int64_t> ids((size_t)num_queries);
  for (int64_t k = 0; k < num_queries; ++k) {
    for (;;) {
      const double dt = at[(size_t)k] - s->now_us();
      if (dt <= 0) break;
      if (dt > 200) std::this_thread::sleep_for(std::chrono::microseconds((int64_t)(dt - 100)));
    }
    const int st = submit_at(s, gs[(size_t)k], rs[(size_t)k], (uint64_t)k, nullptr, at[(size_t)k], true,
                             &ids[(size_t)k]);
    if (st != G500_OK) {  // let the queries already submitted finish, then forget them
      const std::string why = g500_last_error();
      g500_server_drain(s, 600000);
      std::lock_guard<std::mutex> lk(s->mu);
      for (int64_t j = 0; j < k; ++j) s->queries.erase(ids[(size_t)j]);
      return g500::set_error(st, "%s", why.c_str());
    }
  }
  G500_TRY(g500_server_drain(s, 600000));
  std::vector<double> lat;
  lat.reserve((size_t)(num_queries - warmup));
  double first = 1e300, last = 0, sum = 0;
  int64_t failed = 0, nedge = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int64_t k = 0; k < num_queries; ++k) {
      auto it = s->queries.find(ids[(size_t)k]);
      if (it == s->queries.end()) continue;
      const g500_query_result r = it->second.res;
      s->queries.erase(it);
      if (k < warmup) continue;
      if (r.status != G500_OK) {
        ++failed;
        continue;
      }
      const double l = r.done_us - r.arrival_us;
      lat.push_back(l);
      sum += l;
      first = std::min(first, r.arrival_us);
      last = std::max(last, r.done_us);
      nedge += r.nedge;
    }
  }
  memset(rep, 0, sizeof(*rep));
  rep->rate_qps = rate_qps;
  rep->queries = (int64_t)lat.size();
  rep->failed = failed;
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) {
      const size_t i = (size_t)std::min<double>((double)lat.size() - 1, std::ceil(p * (double)lat.size()) - 1);
      return lat[i] * 1e-3;
    };
    rep->p50_ms = pct(0.50);
    rep->p99_ms = pct(0.99);
    rep->mean_ms = sum / (double)lat.size() * 1e-3;
    rep->max_ms = lat.back() * 1e-3;
    rep->wall_s = (last - first) * 1e-6;
    rep->achieved_qps = rep->wall_s > 0 ? (double)lat.size() / rep->wall_s : 0;
    rep->gteps = rep->wall_s > 0 ? (double)nedge / rep->wall_s * 1e-9 : 0;
    rep->nedge = nedge;
  }
  rep->launches = s->launches.load() - l0;
  rep->mean_batch = rep->launches ? (double)(s->lanes_used.load() - q0) / (double)rep->launches : 0;
  rep->max_in_flight = s->max_in_flight.load();
  rep->workers = s->nworkers.load();
  rep->delivery = s->delivery;
  return failed ? g500::set_error(G500_E_DEVICE, "%lld queries failed", (long long)failed) : G500_OK;
}

extern "C" int g500_server_destroy(g500_server* s) {
  if (!s) return G500_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->engine.joinable()) s->engine.join();
  cudaSetDevice(s->device);
  for (auto& ws : s->workers)
    for (Worker& w : ws) {
      if (w.busy) {
        g500_msbfs_wait(w.ms, nullptr);
      }
      g500_msbfs_destroy(w.ms);
    }
  for (auto& ps : s->pworkers)
    for (PlainWorker& w : ps) {
      if (w.busy) g500::bfs_complete(w.bfs, nullptr, nullptr);
      g500_bfs_destroy(w.bfs);
    }
  for (g500_bfs* b : s->plain)
    if (b) g500_bfs_destroy(b);
  if (s->d_pred) cudaFree(s->d_pred);
  if (s->h_pred) cudaFreeHost(s->h_pred);
  free_delivery(s);
  delete s;
  return G500_OK;
}

extern "C" int g500_server_set_delivery(g500_server* s, int mode) {
  if (!s) return g500::set_error(G500_E_INVAL, "null handle");
  if (mode != G500_DELIVER_NONE && mode != G500_DELIVER_DEVICE && mode != G500_DELIVER_HOST)
    return g500::set_error(G500_E_INVAL, "unknown delivery mode %d", mode);
  G500_TRY(g500_server_drain(s, 600000));
  std::lock_guard<std::mutex> lk(s->mu);  // the engine takes slots under this lock
  free_delivery(s);
  if (mode == G500_DELIVER_NONE) return G500_OK;
  G500_CUDA(cudaSetDevice(s->device));
  const int per_graph = s->cfg.max_batch * s->cfg.max_workers_per_graph + 1;  // + a plain run
  const size_t ng = s->graphs.size();
  s->slots.assign(ng, {});
  s->free_slots.assign(ng, {});
  for (size_t g = 0; g < ng; ++g) {
    const size_t bytes = (size_t)std::max<int64_t>(s->graphs[g]->nolv, 1);
    for (int k = 0; k < per_graph; ++k) {
      void* p = nullptr;
      const cudaError_t e = mode == G500_DELIVER_DEVICE ? cudaMalloc(&p, bytes)
                                                        : cudaHostAlloc(&p, bytes, cudaHostAllocDefault);
      if (e != cudaSuccess) {
        cudaGetLastError();
        free_delivery(s);
        return g500::set_error(G500_E_NOMEM, "delivery buffers: %s", cudaGetErrorString(e));
      }
      s->slots[g].push_back(static_cast<uint8_t*>(p));
      s->free_slots[g].push_back(k);
    }
  }
  s->delivery = mode;
  return G500_OK;
}
