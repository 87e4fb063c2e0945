// fvm_server.cu — serving with continuous batching behind the C ABI.
//
// The reference runs one case per process: solve_process
// (src/process/solver_sub.f90:196-207) loops ClassTimeDiscret%solve until
// ClassIteration%converged fires. A server runs that loop for many requests
// at once on one GPU: requests (a case: blocks, boundaries, connections,
// initial state, a number of time steps) are submitted at any time from any
// host thread; a worker thread owned by the server admits them first come,
// first served, into engines whose state arenas are reserved up front (the
// HBM budget), advances every admitted case together (one persistent launch
// per scheme group and RK stage, the captured step graph), and retires a
// case when its steps are done or its residual went non-finite, copying its
// final state to host memory the server owns until the caller releases it.
//
// Cases of different RK stage counts cannot share one engine (their role
// rotations differ), so the server keeps one engine per stage count, each
// with its own stream; their steps are enqueued back to back and overlap on
// the device. Admission counts arena cells over both against the budget.
//
// Threading: submit / poll / wait / fetch / release take the server mutex
// only; every CUDA call happens on the worker thread, which made the device
// current that was current when the server was created.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fvm3d.h"
#include "fvm_engine.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  int64_t id = 0;
  fvm_config cfg;
  std::vector<int64_t> nvert;             // [nblocks][3]
  std::vector<double> dr;                 // [nblocks][3]
  std::vector<std::vector<double>> q;     // initial state, then the result
  std::vector<int32_t> bc;                // [nbc][3]
  std::vector<fvm_connection> conn;
  int64_t steps = 0;
  int64_t cells = 0;                      // arena cells (fvm_block_cells)
  // progress (written by the worker under the mutex)
  int state = FVM_REQ_QUEUED;
  int status = FVM_OK;
  int64_t steps_done = 0;
  double t = 0.0;
  Clock::time_point submitted, finished;
  std::string msg;
  // worker-side placement
  int engine = -1;
  int case_id = -1;
  std::vector<int> blk;
};

}  // namespace

struct fvm_server {
  fvm_server_config cfg;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work;  // worker: a request arrived / stop
  std::condition_variable cv_done;  // fvm_wait: a request finished
  std::map<int64_t, std::shared_ptr<Req>> reqs;
  std::deque<int64_t> queue;
  int64_t next_id = 1;
  bool stop = false;
  std::string err;        // last error of a server call (fvm_server_last_error)
  std::thread worker;
  // worker-only state
  std::unique_ptr<fvm::Engine> eng[2];  // RK3, RK4
  std::vector<std::shared_ptr<Req>> active;
  int64_t active_cells = 0;
  int64_t peak_active_cells = 0;  // written under the mutex
};

namespace {

int set_err(fvm_server* s, int code, const std::string& m) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->err = m;
  return code;
}

// the engine of this stage count, created on first use with the budget reserved
fvm::Engine* engine_for(fvm_server* s, int rk_stages, std::string* why) {
  const int e = rk_stages == 4 ? 1 : 0;
  if (!s->eng[e]) {
    std::unique_ptr<fvm::Engine> en(new fvm::Engine());
    fvm_config c;
    fvm_config_default(&c);
    c.rk_stages = rk_stages;
    int placeholder = -1;
    if (en->add_case(c, &placeholder) || en->remove_case(placeholder) || en->reserve(s->cfg.budget_cells)) {
      *why = en->err;
      return nullptr;
    }
    s->eng[e] = std::move(en);
  }
  return s->eng[e].get();
}

// Place a request's case in its engine and upload its state. Returns
// FVM_OK, FVM_ERR_NOMEM when the reserved arena has no contiguous room now
// (the case is taken out again and the request stays queued), or another
// error (the request fails).
int admit(fvm_server* s, Req& r, std::string* why) {
  fvm::Engine* en = engine_for(s, r.cfg.rk_stages, why);
  if (!en) return FVM_ERR_CUDA;
  int cid = -1;
  int rc = en->add_case(r.cfg, &cid);
  if (rc) {
    *why = en->err;
    return rc;
  }
  const int nb = (int)r.q.size();
  std::vector<int> ids(nb);
  for (int b = 0; b < nb && !rc; ++b) rc = en->add_block(cid, &r.nvert[3 * b], &r.dr[3 * b], &ids[b]);
  for (size_t i = 0; i + 2 < r.bc.size() && !rc; i += 3) rc = en->set_boundary(ids[r.bc[i]], r.bc[i + 1], r.bc[i + 2]);
  for (const auto& c : r.conn) {
    if (rc) break;
    rc = en->connect(ids[c.blk], c.range, ids[c.donor], c.donor_range, c.donor_type);
  }
  if (!rc) {
    std::vector<const double*> qs(nb);
    for (int b = 0; b < nb; ++b) qs[b] = r.q[b].data();
    rc = en->set_states(nb, ids.data(), qs.data());
  }
  if (rc) {
    *why = en->err;
    en->remove_case(cid);
    return rc;
  }
  r.engine = r.cfg.rk_stages == 4 ? 1 : 0;
  r.case_id = cid;
  r.blk = ids;
  return FVM_OK;
}

void finish(fvm_server* s, const std::shared_ptr<Req>& r, int state, int status, const std::string& msg) {
  std::lock_guard<std::mutex> lk(s->mu);
  r->state = state;
  r->status = status;
  r->msg = msg;
  r->finished = Clock::now();
  s->cv_done.notify_all();
}

// Copy a retiring case's final state into its request and free its arena range.
void retire(fvm_server* s, const std::shared_ptr<Req>& r, int state, int status, const std::string& msg) {
  fvm::Engine* en = s->eng[r->engine].get();
  std::vector<double*> qs(r->q.size());
  for (size_t b = 0; b < r->q.size(); ++b) qs[b] = r->q[b].data();
  std::string m = msg;
  if (en->get_states((int)qs.size(), r->blk.data(), qs.data()) && state == FVM_REQ_DONE) {
    state = FVM_REQ_FAILED;
    status = FVM_ERR_CUDA;
    m = en->err;
  }
  en->remove_case(r->case_id);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->active_cells -= r->cells;
  }
  finish(s, r, state, status, m);
}

bool fits(const fvm_server* s, const Req& r) {
  if (s->active_cells + r.cells > s->cfg.budget_cells) return false;
  if (s->cfg.max_active_cells > 0 && !s->active.empty() && s->active_cells + r.cells > s->cfg.max_active_cells)
    return false;
  return true;
}

void worker_main(fvm_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    // -- admit, first come first served, while the head of the queue fits
    std::vector<std::shared_ptr<Req>> take;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty() || !s->active.empty(); });
      if (s->stop) break;
      int64_t cells = s->active_cells;
      const size_t nact = s->active.size();
      for (int64_t id : s->queue) {
        auto& r = s->reqs[id];
        const bool ok = cells + r->cells <= s->cfg.budget_cells &&
                        (s->cfg.max_active_cells <= 0 || (nact == 0 && take.empty()) ||
                         cells + r->cells <= s->cfg.max_active_cells);
        if (!ok) break;
        take.push_back(r);
        cells += r->cells;
      }
    }
    for (auto& r : take) {
      if (!fits(s, *r)) break;
      std::string why;
      const int rc = admit(s, *r, &why);
      if (rc == FVM_ERR_NOMEM && !s->active.empty()) break;  // fragmented arena: wait for a retirement
      std::lock_guard<std::mutex> lk(s->mu);
      s->queue.pop_front();
      if (rc) {
        r->state = FVM_REQ_FAILED;
        r->status = rc;
        r->msg = why;
        r->finished = Clock::now();
        s->cv_done.notify_all();
        continue;
      }
      r->state = FVM_REQ_RUNNING;
      s->active.push_back(r);
      s->active_cells += r->cells;
      s->peak_active_cells = std::max(s->peak_active_cells, s->active_cells);
    }
    if (s->active.empty()) continue;

    // -- advance the running set: a chunk of steps, at most the fewest any
    //    running case still needs, on every engine that holds one
    int64_t k = s->cfg.chunk_steps;
    for (auto& r : s->active) k = std::min(k, r->steps - r->steps_done);
    bool used[2] = {false, false};
    for (auto& r : s->active) used[r->engine] = true;
    int rc[2] = {FVM_OK, FVM_OK};
    for (int e = 0; e < 2; ++e)
      if (used[e]) rc[e] = s->eng[e]->step((int)k);
    for (int e = 0; e < 2; ++e)
      if (used[e] && !rc[e] && cudaStreamSynchronize(s->eng[e]->stream) != cudaSuccess) {
        rc[e] = FVM_ERR_CUDA;
        s->eng[e]->err = cudaGetErrorString(cudaGetLastError());
      }
    // -- progress (one copy of every case state per engine), and retire
    //    what is done or failed
    std::vector<fvm::DevCaseState> states[2];
    for (int e = 0; e < 2; ++e)
      if (used[e] && !rc[e]) rc[e] = s->eng[e]->read_all_case_states(&states[e]);
    std::vector<std::shared_ptr<Req>> keep;
    for (auto& r : s->active) {
      fvm::Engine* en = s->eng[r->engine].get();
      if (rc[r->engine]) {
        retire(s, r, FVM_REQ_FAILED, rc[r->engine], en->err);
        continue;
      }
      fvm::DevCaseState cs;
      std::memset(&cs, 0, sizeof cs);
      int rr = FVM_OK;
      if (r->case_id < (int)states[r->engine].size() && en->has_case_state(r->case_id))
        cs = states[r->engine][r->case_id];
      else
        rr = en->read_case_state(r->case_id, &cs);
      {
        std::lock_guard<std::mutex> lk(s->mu);
        r->steps_done += k;
        if (!rr) r->t = cs.t;
      }
      if (rr) {
        retire(s, r, FVM_REQ_FAILED, rr, en->err);
      } else if (cs.status) {
        retire(s, r, FVM_REQ_FAILED, cs.status,
               cs.status == FVM_ERR_NONFINITE ? "Error: ABSRES NaN" : "Error: Absolute Residual Exceeds Threshold 1E10.");
      } else if (r->steps_done >= r->steps) {
        retire(s, r, FVM_REQ_DONE, FVM_OK, "");
      } else {
        keep.push_back(r);
      }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->active.swap(keep);
  }
  // shutting down: running cases end as failed, the engines go with the server
  for (auto& r : s->active) finish(s, r, FVM_REQ_FAILED, FVM_ERR_STATE, "server destroyed");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->active.clear();
  }
  for (auto& e : s->eng) e.reset();
}

}  // namespace

extern "C" {

int fvm_server_config_default(fvm_server_config* c) {
  if (!c) return FVM_ERR_INVALID;
  std::memset(c, 0, sizeof *c);
  c->struct_size = (int32_t)sizeof(fvm_server_config);
  c->chunk_steps = 8;
  c->budget_cells = (int64_t)1 << 24;
  c->max_active_cells = 0;
  c->max_queued = 1024;
  return FVM_OK;
}

int fvm_server_create(const fvm_server_config* cfg, fvm_server** out) {
  if (!cfg || !out) return FVM_ERR_INVALID;
  *out = nullptr;
  if (cfg->struct_size != (int32_t)sizeof(fvm_server_config) || cfg->chunk_steps < 1 || cfg->budget_cells < 1 ||
      cfg->max_active_cells < 0 || cfg->max_queued < 1)
    return FVM_ERR_INVALID;
  fvm_server* s = new (std::nothrow) fvm_server();
  if (!s) return FVM_ERR_NOMEM;
  s->cfg = *cfg;
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return FVM_ERR_CUDA;
  }
  try {
    s->worker = std::thread(worker_main, s);
  } catch (...) {
    delete s;
    return FVM_ERR_NOMEM;
  }
  *out = s;
  return FVM_OK;
}

int fvm_case_submit(fvm_server* s, const fvm_request* r, int64_t* request_id) {
  if (!s) return FVM_ERR_INVALID;
  if (!r || !request_id || r->struct_size != (int32_t)sizeof(fvm_request) || !r->cfg)
    return set_err(s, FVM_ERR_INVALID, "null request or struct_size mismatch");
  if (r->nblocks < 1 || !r->nvert || !r->dr || !r->q)
    return set_err(s, FVM_ERR_INVALID, "a request needs nblocks >= 1 with nvert, dr and q");
  if (r->steps < 1) return set_err(s, FVM_ERR_INVALID, "steps must be >= 1");
  if ((r->nbc > 0 && !r->bc) || (r->nconn > 0 && !r->conn) || r->nbc < 0 || r->nconn < 0)
    return set_err(s, FVM_ERR_INVALID, "bc / conn arrays missing");
  if (r->cfg->struct_size != (int32_t)sizeof(fvm_config))
    return set_err(s, FVM_ERR_INVALID, "fvm_config.struct_size mismatch");
  auto q = std::make_shared<Req>();
  q->cfg = *r->cfg;
  q->steps = r->steps;
  q->nvert.assign(r->nvert, r->nvert + 3 * r->nblocks);
  q->dr.assign(r->dr, r->dr + 3 * r->nblocks);
  for (int b = 0; b < r->nblocks; ++b) {
    const int64_t* n = &q->nvert[3 * b];
    int64_t c = 0;
    if (fvm_block_cells(q->cfg.idimension, n, &c) || !r->q[b])
      return set_err(s, FVM_ERR_INVALID, "bad block shape or null state");
    q->cells += c;
    const size_t vals = (size_t)5 * n[0] * n[1] * n[2];
    q->q.emplace_back(r->q[b], r->q[b] + vals);
  }
  for (int i = 0; i < r->nbc; ++i) {
    const int32_t* b = r->bc + 3 * i;
    if (b[0] < 0 || b[0] >= r->nblocks) return set_err(s, FVM_ERR_INVALID, "bc block index out of range");
    q->bc.insert(q->bc.end(), b, b + 3);
  }
  for (int i = 0; i < r->nconn; ++i) {
    const fvm_connection& c = r->conn[i];
    if (c.blk < 0 || c.blk >= r->nblocks || c.donor < 0 || c.donor >= r->nblocks)
      return set_err(s, FVM_ERR_INVALID, "connection block index out of range");
    q->conn.push_back(c);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (q->cells > s->cfg.budget_cells) {
    s->err = "the request needs more arena cells than the whole budget";
    return FVM_ERR_INVALID;
  }
  if ((int64_t)s->queue.size() >= s->cfg.max_queued) {
    s->err = "the queue is full";
    return FVM_ERR_BUSY;
  }
  q->id = s->next_id++;
  q->submitted = Clock::now();
  s->reqs[q->id] = q;
  s->queue.push_back(q->id);
  *request_id = q->id;
  s->cv_work.notify_one();
  return FVM_OK;
}

int fvm_poll(fvm_server* s, int64_t request_id, int* state, int64_t* steps_done, double* t, double* latency_s,
             int* status) {
  if (!s) return FVM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) {
    s->err = "unknown or released request id";
    return FVM_ERR_NOT_FOUND;
  }
  const Req& r = *it->second;
  if (state) *state = r.state;
  if (steps_done) *steps_done = r.steps_done;
  if (t) *t = r.t;
  if (status) *status = r.status;
  if (latency_s) {
    const bool end = r.state == FVM_REQ_DONE || r.state == FVM_REQ_FAILED;
    *latency_s = std::chrono::duration<double>((end ? r.finished : Clock::now()) - r.submitted).count();
  }
  if (r.state == FVM_REQ_FAILED) s->err = r.msg;
  return FVM_OK;
}

int fvm_wait(fvm_server* s, int64_t request_id, double timeout_s, int* state) {
  if (!s) return FVM_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) {
    s->err = "unknown or released request id";
    return FVM_ERR_NOT_FOUND;
  }
  std::shared_ptr<Req> r = it->second;
  const auto done = [&] { return r->state == FVM_REQ_DONE || r->state == FVM_REQ_FAILED; };
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 0.0), done);
  if (state) *state = r->state;
  if (!ok) {
    s->err = "the request did not finish within the timeout";
    return FVM_ERR_TIMEOUT;
  }
  return FVM_OK;
}

int fvm_fetch_state(fvm_server* s, int64_t request_id, int blk, double* q) {
  if (!s || !q) return FVM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) {
    s->err = "unknown or released request id";
    return FVM_ERR_NOT_FOUND;
  }
  const Req& r = *it->second;
  if (r.state != FVM_REQ_DONE && r.state != FVM_REQ_FAILED) {
    s->err = "the request has not finished";
    return FVM_ERR_BUSY;
  }
  if (blk < 0 || blk >= (int)r.q.size()) {
    s->err = "block index out of range";
    return FVM_ERR_INVALID;
  }
  std::memcpy(q, r.q[blk].data(), sizeof(double) * r.q[blk].size());
  return FVM_OK;
}

int fvm_release(fvm_server* s, int64_t request_id) {
  if (!s) return FVM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) {
    s->err = "unknown or released request id";
    return FVM_ERR_NOT_FOUND;
  }
  if (it->second->state != FVM_REQ_DONE && it->second->state != FVM_REQ_FAILED) {
    s->err = "the request has not finished";
    return FVM_ERR_BUSY;
  }
  s->reqs.erase(it);
  return FVM_OK;
}

int fvm_server_stats(fvm_server* s, int64_t* active_cells, int64_t* peak_active_cells, int* running, int* queued) {
  if (!s) return FVM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  if (active_cells) *active_cells = s->active_cells;
  if (peak_active_cells) *peak_active_cells = s->peak_active_cells;
  if (running) *running = (int)s->active.size();
  if (queued) *queued = (int)s->queue.size();
  return FVM_OK;
}

int fvm_server_last_error(fvm_server* s, char* buf, size_t n) {
  if (!s || !buf || n == 0) return FVM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  std::snprintf(buf, n, "%s", s->err.c_str());
  return FVM_OK;
}

int fvm_server_destroy(fvm_server* s) {
  if (!s) return FVM_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
  return FVM_OK;
}

}  // extern "C"
