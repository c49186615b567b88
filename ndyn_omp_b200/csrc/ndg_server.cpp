// ndg_server.cpp -- the serving loop: continuous batching of independent MD
// runs on one GPU (no counterpart in the reference, which runs one system
// per process).
//
// A server owns one context.  Submitted requests wait in a host queue with
// copies of their arrays.  Each ndg_server_step
//   1. admits queued requests, in submission order, whose estimated device
//      bytes fit what the resident runs leave of the HBM budget (a request
//      that does not fit keeps its place; later smaller ones may pass it),
//   2. adds them as systems of the context and runs the dynamics prologue
//      (cells + lists) for them alone,
//   3. advances every resident run by one block of up to block_steps steps:
//      one graph launch for all of them (k_begin_block gives each run its
//      share, runs that end inside the block go idle for the rest of it),
//   4. retires runs whose last step is done: applies their pending velocity
//      scale, copies their final state to host memory and frees their
//      device ranges for the next admissions.
// Runs never wait for each other: a request that arrives while others are
// on the GPU joins at the next block.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "../../include/ndyn_gpu.h"
#include "ndg_internal.h"

namespace {

struct Request {
  long long ticket = 0;
  int status = 0;  // 0 queued, 1 resident, 2 done, <0 failed (NDG_ERR_*)
  int np = 0, ntypes = 0, npairs = 0, ptsize = 0;
  double ptrmin = 0.25;
  std::vector<double> mass, rcpair, ppair, fpair, pos, vel;
  std::vector<int> pairmat, typ;
  std::vector<int> spring;         // spring pairs (empty: none)
  std::vector<double> pair_params;  // their PairParams, 4 per pair
  double box[3] = {0, 0, 0};
  ndg_control ctl{};
  int nsteps = 0, left = 0;
  long long bytes = 0;
  int sys = -1;
  std::vector<ndg_thermo> rows;
  std::vector<double> rpos, rvel, racc;
  double rbox[3] = {0, 0, 0};
};

long long estimate_bytes(const Request &r, int precision) {
  const double vol = r.box[0] * r.box[1] * r.box[2];
  double rc = 0.0;
  for (double x : r.rcpair) rc = std::max(rc, x);
  const double skin = r.ctl.skin < 0 ? 0.2 * rc : r.ctl.skin;
  return ndg_system_bytes(r.np, r.ntypes, r.npairs, r.ptsize, vol > 0 ? r.np / vol : 0.1,
                          rc + skin, precision);
}

}  // namespace

struct ndg_server {
  ndg_ctx *ctx = nullptr;
  int precision = NDG_PREC_MIXED;
  long long budget = 0, in_use = 0;
  int block = 100;
  long long next_ticket = 1;
  std::deque<long long> queue;
  std::map<long long, Request> reqs;
  std::map<int, long long> by_sys;  // resident system -> ticket
  std::vector<long long> finished;  // not yet polled
  int completed = 0, failed = 0;
  double atom_steps = 0.0;
  double t_admit = 0, t_setup = 0, t_block = 0, t_retire = 0;
  int blocks = 0;
};

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

void thermo_sink(const ndg_thermo *t, void *user) {
  ndg_server *s = static_cast<ndg_server *>(user);
  auto it = s->by_sys.find(t->sys);
  if (it == s->by_sys.end()) return;
  auto r = s->reqs.find(it->second);
  if (r != s->reqs.end()) r->second.rows.push_back(*t);
}

void fail(ndg_server *s, Request &r, int status) {
  if (r.sys >= 0) {
    ndg_remove_system(s->ctx, r.sys);
    s->by_sys.erase(r.sys);
    s->in_use -= r.bytes;
    r.sys = -1;
  }
  r.status = status < 0 ? status : NDG_ERR_CUDA;
  s->failed += 1;
  s->finished.push_back(r.ticket);
}

// copy a finished run's state out and give its device ranges back
int retire(ndg_server *s, Request &r) {
  int rc = ndg_internal::flush_system(s->ctx, r.sys);
  if (rc) return rc;
  r.rpos.resize(3 * (size_t)r.np);
  r.rvel.resize(3 * (size_t)r.np);
  r.racc.resize(3 * (size_t)r.np);
  rc = ndg_get_state(s->ctx, r.sys, r.rpos.data(), r.rvel.data(), r.racc.data(), r.rbox);
  if (rc) return rc;
  rc = ndg_remove_system(s->ctx, r.sys);
  s->by_sys.erase(r.sys);
  s->in_use -= r.bytes;
  r.sys = -1;
  r.status = 2;
  s->completed += 1;
  s->finished.push_back(r.ticket);
  // host copies of the inputs are no longer needed
  r.pos.clear();
  r.vel.clear();
  r.pos.shrink_to_fit();
  r.vel.shrink_to_fit();
  return rc;
}

}  // namespace

extern "C" {

int ndg_admit_plan(const long long *bytes, int n, long long budget, long long in_use, int *admit) {
  if (n < 0 || (n > 0 && (!bytes || !admit))) return NDG_ERR_ARG;
  int k = 0;
  long long used = in_use;
  for (int q = 0; q < n; ++q) {
    admit[q] = 0;
    if (bytes[q] >= 0 && used + bytes[q] <= budget) {
      admit[q] = 1;
      used += bytes[q];
      ++k;
    }
  }
  return k;
}

int ndg_server_create(ndg_server **out, int device, int precision, long long budget,
                      int block_steps) {
  if (!out || budget <= 0 || block_steps < 1) return NDG_ERR_ARG;
  *out = nullptr;
  ndg_ctx *ctx = nullptr;
  int rc = ndg_create(&ctx, device, precision);
  if (rc) return rc;
  rc = ndg_set_tuning(ctx, 0, block_steps);
  if (rc) {
    ndg_destroy(ctx);
    return rc;
  }
  ndg_server *s = new ndg_server();
  s->ctx = ctx;
  s->precision = precision;
  s->budget = budget;
  s->block = block_steps;
  *out = s;
  return NDG_OK;
}

int ndg_server_destroy(ndg_server *s) {
  if (!s) return NDG_ERR_ARG;
  ndg_destroy(s->ctx);
  delete s;
  return NDG_OK;
}

int ndg_server_context(ndg_server *s, ndg_ctx **ctx) {
  if (!s || !ctx) return NDG_ERR_ARG;
  *ctx = s->ctx;
  return NDG_OK;
}

int ndg_server_submit(ndg_server *s, const ndg_request *q, long long *ticket) {
  if (!s || !q || q->np < 1 || q->ntypes < 1 || q->npairs < 1 || q->ptsize < 2 || q->nsteps < 1 ||
      !q->mass || !q->pairmat || !q->rcpair || !q->ppair || !q->fpair || !q->typ || !q->pos ||
      !q->box)
    return NDG_ERR_ARG;
  Request r;
  r.ticket = s->next_ticket++;
  r.np = q->np;
  r.ntypes = q->ntypes;
  r.npairs = q->npairs;
  r.ptsize = q->ptsize;
  r.ptrmin = q->ptrmin;
  r.mass.assign(q->mass, q->mass + q->ntypes);
  r.pairmat.assign(q->pairmat, q->pairmat + q->ntypes * q->ntypes);
  r.rcpair.assign(q->rcpair, q->rcpair + q->npairs);
  const size_t T = (size_t)(q->ptsize + 1) * q->npairs;
  r.ppair.assign(q->ppair, q->ppair + T);
  r.fpair.assign(q->fpair, q->fpair + T);
  r.typ.assign(q->typ, q->typ + q->np);
  r.pos.assign(q->pos, q->pos + 3 * (size_t)q->np);
  if (q->vel) r.vel.assign(q->vel, q->vel + 3 * (size_t)q->np);
  if (q->spring) {
    if (!q->pair_params) return NDG_ERR_ARG;
    r.spring.assign(q->spring, q->spring + q->npairs);
    r.pair_params.assign(q->pair_params, q->pair_params + 4 * (size_t)q->npairs);
  }
  for (int d = 0; d < 3; ++d) r.box[d] = q->box[d];
  r.ctl = q->control;
  r.nsteps = r.left = q->nsteps;
  r.bytes = estimate_bytes(r, s->precision);
  if (r.bytes > s->budget) return NDG_ERR_BUDGET;  // could never be admitted
  const long long t = r.ticket;
  s->reqs.emplace(t, std::move(r));
  s->queue.push_back(t);
  if (ticket) *ticket = t;
  return NDG_OK;
}

int ndg_server_step(ndg_server *s, int *completed) {
  if (!s) return NDG_ERR_ARG;
  const int done0 = s->completed + s->failed;
  double t = now_s();
  // 1. admission by HBM budget, in queue order
  std::vector<long long> bytes;
  for (long long t : s->queue) bytes.push_back(s->reqs[t].bytes);
  std::vector<int> admit(bytes.size(), 0);
  ndg_admit_plan(bytes.data(), (int)bytes.size(), s->budget, s->in_use, admit.data());
  std::deque<long long> waiting;
  std::vector<int> fresh;
  std::vector<long long> fresh_t;
  {
    // room for the whole batch at once (a system's atoms are padded to 256)
    long long atoms = 0;
    for (size_t k = 0; k < s->queue.size(); ++k)
      if (admit[k]) atoms += (s->reqs[s->queue[k]].np + 255) / 256 * 256;
    if (atoms) ndg_internal::reserve_atoms(s->ctx, atoms);  // a failure shows in the adds
  }
  for (size_t k = 0; k < s->queue.size(); ++k) {
    const long long t = s->queue[k];
    if (!admit[k]) {
      waiting.push_back(t);
      continue;
    }
    Request &r = s->reqs[t];
    int sys = -1;
    int rc = ndg_add_system(s->ctx, r.np, r.ntypes, r.npairs, r.ptsize, r.ptrmin, r.mass.data(),
                            r.pairmat.data(), r.rcpair.data(), r.ppair.data(), r.fpair.data(),
                            r.typ.data(), r.pos.data(), r.vel.empty() ? nullptr : r.vel.data(),
                            nullptr, r.box, &sys);
    if (!rc) rc = ndg_set_control(s->ctx, sys, &r.ctl);
    if (!rc && !r.spring.empty())
      rc = ndg_set_springs(s->ctx, sys, r.spring.data(), r.pair_params.data());
    if (rc) {
      if (sys >= 0) ndg_remove_system(s->ctx, sys);
      r.status = rc;
      s->failed += 1;
      s->finished.push_back(t);
      continue;
    }
    r.sys = sys;
    r.status = 1;
    s->by_sys[sys] = t;
    s->in_use += r.bytes;
    fresh.push_back(sys);
    fresh_t.push_back(t);
  }
  s->queue.swap(waiting);
  {
    const double t1 = now_s();
    s->t_admit += t1 - t;
    t = t1;
  }
  // 2. prologue for the new runs only (if the joint build fails, one at a
  // time, so that only the runs that cannot start fail)
  if (!fresh.empty()) {
    if (ndg_internal::setup_systems(s->ctx, fresh) != NDG_OK) {
      for (size_t k = 0; k < fresh.size(); ++k) {
        const int rc = ndg_internal::setup_systems(s->ctx, {fresh[k]});
        if (rc) fail(s, s->reqs[fresh_t[k]], rc);
      }
    }
    for (size_t k = 0; k < fresh.size(); ++k) {
      Request &r = s->reqs[fresh_t[k]];
      if (r.status == 1) ndg_internal::arm_built(s->ctx, r.sys, r.nsteps);
    }
  }
  {
    const double t1 = now_s();
    s->t_setup += t1 - t;
    t = t1;
  }
  // 3. one block for every resident run
  if (!s->by_sys.empty()) {
    int rc = ndg_internal::run_block(s->ctx, s->block, thermo_sink, s);
    s->blocks += 1;
    {
      const double t1 = now_s();
      s->t_block += t1 - t;
      t = t1;
    }
    std::vector<long long> resident;
    for (auto &kv : s->by_sys) resident.push_back(kv.second);
    if (rc && rc != NDG_ERR_NEIMAX && rc != NDG_ERR_OUT_OF_BOX && rc != NDG_ERR_CELLS) return rc;
    for (long long t : resident) {
      Request &r = s->reqs[t];
      if (rc) {
        int err = 0;
        ndg_internal::take_system_error(s->ctx, r.sys, &err);
        if (err) {
          fail(s, r, (err & 1) ? NDG_ERR_NEIMAX : (err & 2) ? NDG_ERR_OUT_OF_BOX : NDG_ERR_CELLS);
          continue;
        }
      }
      const int k = std::min(r.left, s->block);
      r.left -= k;
      s->atom_steps += (double)r.np * k;
      // 4. retire finished runs
      if (r.left == 0) {
        int e = retire(s, r);
        if (e) fail(s, r, e);
      }
    }
  }
  s->t_retire += now_s() - t;
  if (completed) *completed = s->completed + s->failed - done0;
  return NDG_OK;
}

int ndg_server_poll(ndg_server *s, long long *tickets, int cap, int *n) {
  if (!s || !n || (cap > 0 && !tickets)) return NDG_ERR_ARG;
  const int m = std::min(cap, (int)s->finished.size());
  for (int k = 0; k < m; ++k) tickets[k] = s->finished[k];
  s->finished.erase(s->finished.begin(), s->finished.begin() + m);
  *n = m;
  return NDG_OK;
}

int ndg_server_status(ndg_server *s, long long ticket, int *status) {
  if (!s || !status) return NDG_ERR_ARG;
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return NDG_ERR_NOT_FOUND;
  *status = it->second.status;
  return NDG_OK;
}

int ndg_server_result(ndg_server *s, long long ticket, double *pos, double *vel, double *acc,
                      double *box, ndg_thermo *rows, int cap, int *nrows) {
  if (!s) return NDG_ERR_ARG;
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return NDG_ERR_NOT_FOUND;
  Request &r = it->second;
  if (r.status < 0) {
    const int st = r.status;
    s->reqs.erase(it);
    return st;
  }
  if (r.status != 2) return NDG_ERR_ARG;  // not finished yet
  const size_t n3 = 3 * (size_t)r.np;
  if (pos) std::memcpy(pos, r.rpos.data(), n3 * sizeof(double));
  if (vel) std::memcpy(vel, r.rvel.data(), n3 * sizeof(double));
  if (acc) std::memcpy(acc, r.racc.data(), n3 * sizeof(double));
  if (box)
    for (int d = 0; d < 3; ++d) box[d] = r.rbox[d];
  const int m = std::min(cap, (int)r.rows.size());
  if (rows && m > 0) std::memcpy(rows, r.rows.data(), (size_t)m * sizeof(ndg_thermo));
  if (nrows) *nrows = (int)r.rows.size();
  s->reqs.erase(it);
  return NDG_OK;
}

int ndg_server_stats_get(ndg_server *s, ndg_server_stats *st) {
  if (!s || !st) return NDG_ERR_ARG;
  st->queued = (int)s->queue.size();
  st->resident = (int)s->by_sys.size();
  st->completed = s->completed;
  st->failed = s->failed;
  st->bytes_in_use = s->in_use;
  st->budget = s->budget;
  st->atom_steps = s->atom_steps;
  st->t_admit = s->t_admit;
  st->t_setup = s->t_setup;
  st->t_block = s->t_block;
  st->t_retire = s->t_retire;
  st->graph_captures = ndg_internal::graph_captures(s->ctx);
  st->blocks = s->blocks;
  return NDG_OK;
}

}  // extern "C"
