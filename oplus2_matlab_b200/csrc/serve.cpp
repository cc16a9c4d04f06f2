// serve.cpp -- the continuous-batching solve server (include/op2b_serve.h):
// request queue, admission under a memory budget and a cap, retirement of
// stopped solves, and the latency record, over a group of solves reached
// through a table of functions (the GPU engine of group.cu, or a stand-in).

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "internal.h"
#include "op2b_serve.h"

namespace {

struct Req {
  long long rid = 0;
  op2b_mesh mesh;  // the caller's arrays, valid until admission
  double mach = 0, alpha = 0, rel_tol = 0;
  int max_iter = 0;
  double arrival = 0, admitted = -1, finished = -1;
  int sid = -1, iterations = 0;
};

struct Result {
  std::vector<double> rms;
  std::vector<unsigned char> q;
};

}  // namespace

struct op2b_server_s {
  op2b_group_ops ops;
  long long budget = 0;
  int k = 10, max_active = 0, policy = 0, keep_q = 0, real_bytes = 4;
  bool unsorted = false;
  std::deque<Req> queue;
  std::map<int, Req> active;           // by solve id
  std::vector<Req> done;               // every finished request
  size_t reported = 0;                 // done[0, reported) returned by op2b_server_done
  std::map<long long, Result> results;  // kept until released
  int peak = 0;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() {
    if (ops.now) return ops.now(ops.ctx);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  bool admit(double t) {
    if (policy == 1 && unsorted && queue.size() > 1)
      std::stable_sort(queue.begin(), queue.end(), [](const Req &a, const Req &b) {
        const double wa = (double)a.mesh.ncell * a.max_iter, wb = (double)b.mesh.ncell * b.max_iter;
        return wa != wb ? wa < wb : a.arrival < b.arrival;
      });
    unsorted = false;
    while (!queue.empty()) {
      if (max_active > 0 && (int)active.size() >= max_active) break;
      Req &r = queue.front();
      const long long need = ops.solve_bytes(ops.ctx, r.rid, &r.mesh, r.max_iter);
      if (!active.empty() && ops.device_bytes(ops.ctx) + need > budget) break;
      const int sid =
          ops.add(ops.ctx, r.rid, &r.mesh, r.mach, r.alpha, r.max_iter, r.rel_tol);
      if (sid < 0) return false;
      Req a = r;
      queue.pop_front();
      a.sid = sid;
      a.admitted = t;
      // the caller's arrays may go now: keep only the sizes
      a.mesh.cell = a.mesh.edge = a.mesh.ecell = a.mesh.bedge = a.mesh.becell = a.mesh.bound =
          nullptr;
      a.mesh.x64 = nullptr;
      a.mesh.x32 = nullptr;
      active[sid] = a;
    }
    peak = std::max(peak, (int)active.size());
    return true;
  }
};

using op2b::fail;

namespace {

// the GPU engine's table
int g_add(void *ctx, long long, const op2b_mesh *m, double mach, double alpha, int max_iter,
          double rel_tol) {
  return op2b_group_add((op2b_group)ctx, m, mach, alpha, max_iter, rel_tol);
}
int g_run(void *ctx, int niter) { return op2b_group_run((op2b_group)ctx, niter); }
int g_poll(void *ctx, int *ids, int max) { return op2b_group_poll((op2b_group)ctx, ids, max); }
int g_history(void *ctx, int sid, double *rms, int max) {
  return op2b_group_history((op2b_group)ctx, sid, rms, max);
}
int g_fetch_q(void *ctx, int sid, void *q) { return op2b_group_fetch_q((op2b_group)ctx, sid, q); }
int g_remove(void *ctx, int sid) { return op2b_group_remove((op2b_group)ctx, sid); }
long long g_solve_bytes(void *ctx, long long, const op2b_mesh *m, int max_iter) {
  return op2b_group_solve_bytes((op2b_group)ctx, m->nnode, m->ncell, m->nedge, m->nbedge,
                                max_iter);
}
long long g_device_bytes(void *ctx) { return op2b_group_device_bytes((op2b_group)ctx); }

}  // namespace

extern "C" {

int op2b_group_ops_fill(op2b_group g, op2b_group_ops *ops) {
  if (!g || !ops) return -1;
  memset(ops, 0, sizeof *ops);
  ops->ctx = g;
  ops->add = g_add;
  ops->run = g_run;
  ops->poll = g_poll;
  ops->history = g_history;
  ops->fetch_q = g_fetch_q;
  ops->remove = g_remove;
  ops->solve_bytes = g_solve_bytes;
  ops->device_bytes = g_device_bytes;
  ops->now = nullptr;
  return 0;
}

op2b_server op2b_server_create(const op2b_group_ops *ops, long long budget_bytes,
                               int iters_per_step, int max_active, int policy, int keep_q,
                               int real_bytes) {
  if (!ops || !ops->add || !ops->run || !ops->poll || !ops->history || !ops->remove ||
      !ops->solve_bytes || !ops->device_bytes || (keep_q && !ops->fetch_q) ||
      iters_per_step < 1 || (policy != 0 && policy != 1) ||
      (real_bytes != 4 && real_bytes != 8)) {
    fail(-1, "op2b_server_create error: incomplete group table or bad arguments\n");
    return nullptr;
  }
  op2b_server s = new op2b_server_s();
  s->ops = *ops;
  s->budget = budget_bytes;
  s->k = iters_per_step;
  s->max_active = max_active;
  s->policy = policy;
  s->keep_q = keep_q;
  s->real_bytes = real_bytes;
  return s;
}

void op2b_server_destroy(op2b_server s) { delete s; }

int op2b_server_submit(op2b_server s, long long rid, const op2b_mesh *m, double mach,
                       double alpha_deg, int max_iter, double rel_tol, double arrival) {
  if (!s || !m || max_iter < 1 || m->ncell < 0) return -1;
  Req r;
  r.rid = rid;
  r.mesh = *m;
  r.mach = mach;
  r.alpha = alpha_deg;
  r.max_iter = max_iter;
  r.rel_tol = rel_tol;
  r.arrival = arrival;
  s->queue.push_back(r);
  s->unsorted = true;
  return 0;
}

int op2b_server_step(op2b_server s) {
  if (!s) return -1;
  if (s->active.empty() && !s->admit(s->now())) return -1;
  if (s->active.empty()) return 0;
  if (s->ops.run(s->ops.ctx, s->k) < 0) return -1;
  if (!s->admit(s->now())) return -1;  // uploads overlap the iterations just enqueued
  std::vector<int> ids(std::max<size_t>(16, s->active.size()));
  const int n = s->ops.poll(s->ops.ctx, ids.data(), (int)ids.size());
  if (n < 0) return -1;
  const double t = s->now();
  int finished = 0;
  for (int i = 0; i < n; i++) {
    auto it = s->active.find(ids[i]);
    if (it == s->active.end()) continue;
    Req r = it->second;
    s->active.erase(it);
    r.finished = t;
    Result &res = s->results[r.rid];
    res.rms.assign((size_t)r.max_iter, 0.0);
    const int got = s->ops.history(s->ops.ctx, r.sid, res.rms.data(), r.max_iter);
    if (got < 0) return -1;
    res.rms.resize((size_t)got);
    r.iterations = got;
    if (s->keep_q) {
      res.q.assign((size_t)r.mesh.ncell * 4 * s->real_bytes, 0);
      if (s->ops.fetch_q(s->ops.ctx, r.sid, res.q.data()) < 0) return -1;
    }
    if (s->ops.remove(s->ops.ctx, r.sid) < 0) return -1;
    s->done.push_back(r);
    finished++;
  }
  return finished;
}

int op2b_server_done(op2b_server s, op2b_served *out, int max) {
  if (!s || (!out && max > 0)) return -1;
  int n = 0;
  while (s->reported < s->done.size() && n < max) {
    const Req &r = s->done[s->reported++];
    out[n++] = op2b_served{r.rid, r.sid, r.iterations, r.arrival, r.admitted, r.finished};
  }
  return n;
}

int op2b_server_history(op2b_server s, long long rid, double *rms, int max) {
  if (!s) return -1;
  auto it = s->results.find(rid);
  if (it == s->results.end()) return -1;
  const int n = std::min(max, (int)it->second.rms.size());
  if (n > 0) memcpy(rms, it->second.rms.data(), sizeof(double) * (size_t)n);
  return (int)it->second.rms.size();
}

int op2b_server_q(op2b_server s, long long rid, void *q) {
  if (!s || !q) return -1;
  auto it = s->results.find(rid);
  if (it == s->results.end() || it->second.q.empty()) return -1;
  memcpy(q, it->second.q.data(), it->second.q.size());
  return 0;
}

void op2b_server_release(op2b_server s, long long rid) {
  if (s) s->results.erase(rid);
}

int op2b_server_active(op2b_server s, long long *rids, int *sids, int max) {
  if (!s) return -1;
  int n = 0;
  for (auto &kv : s->active) {
    if (n < max) {
      if (rids) rids[n] = kv.second.rid;
      if (sids) sids[n] = kv.first;
    }
    n++;
  }
  return n;
}

int op2b_server_queued(op2b_server s) { return s ? (int)s->queue.size() : -1; }
int op2b_server_peak_active(op2b_server s) { return s ? s->peak : -1; }
int op2b_server_idle(op2b_server s) { return s && s->queue.empty() && s->active.empty(); }
double op2b_server_now(op2b_server s) { return s ? s->now() : 0.0; }

int op2b_server_latency(op2b_server s, double *p50, double *p99, double *mean, double *max) {
  if (!s || s->done.empty()) return -1;
  std::vector<double> lat;
  lat.reserve(s->done.size());
  double sum = 0;
  for (const Req &r : s->done) {
    lat.push_back(r.finished - r.arrival);
    sum += lat.back();
  }
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double p) {
    const double x = p / 100.0 * (double)(lat.size() - 1);
    const size_t lo = (size_t)floor(x);
    const size_t hi = std::min(lo + 1, lat.size() - 1);
    return lat[lo] + (x - (double)lo) * (lat[hi] - lat[lo]);
  };
  if (p50) *p50 = pct(50.0);
  if (p99) *p99 = pct(99.0);
  if (mean) *mean = sum / (double)lat.size();
  if (max) *max = lat.back();
  return 0;
}

}  // extern "C"
