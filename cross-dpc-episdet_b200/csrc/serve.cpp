// Request server with continuous batching (include/epik2.h, "Serving form").
//
// Host C++ on top of the public C ABI only: one epik2 context, one worker thread.  The
// worker repeats: admit queued scans while the launch's work target, its slot limit and
// free device memory above the reserve allow, taking one scan per pending request in
// turn (round robin from where the previous round stopped, so a small request is not held
// behind a large one); create each admitted scan's dataset (a replicate sharing a
// resident genotype matrix, or a freshly uploaded matrix); run one batched launch over
// all of them (epik2_scan_batch) -- except that three or more replicates of one resident matrix
// admitted together run in the replicate form (epik2_scan_replicates: each tile's all-sample
// counts shared by them); release the datasets; and complete the requests whose scans are
// all done.  Requests that arrive during a launch join the next admission
// round.  Submitting never waits for the device: it copies the request and queues it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/epik2.h"

namespace {

using Clock = std::chrono::steady_clock;

enum { kPending = 0, kDone = 1 };

struct Request {
  int64_t id = 0;
  int32_t dataset = -1;        // resident genotype owner (replicates) or -1 (fresh matrix)
  int64_t n_samples = 0, n_snps = 0;
  int32_t n_scans = 0;
  int32_t n_admitted = 0;       // scans handed to a launch (or finished unlaunched)
  std::vector<uint8_t> phenos;  // n_scans x n_samples
  std::vector<uint8_t> geno;    // fresh matrix only
  std::vector<epik2_best> results;
  int32_t n_done = 0, n_failed = 0;
  int state = kPending;
  int status = EPIK2_OK;
  bool cancelled = false;
  Clock::time_point t_submit, t_done;
};

struct Item {
  Request* req;
  int32_t scan;
};

struct Matrix {
  int32_t dataset;
  int64_t n_samples, n_snps;
};

double work_of(int64_t s, int64_t m) { return (double)m * (double)(m - 1) * (double)(m - 2) / 6.0 * (double)s; }

}  // namespace

struct epik2_server {
  epik2_ctx* ctx = nullptr;
  epik2_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  std::map<int32_t, Matrix> matrices;  // matrix id -> resident dataset
  std::map<int64_t, std::unique_ptr<Request>> requests;
  std::deque<Request*> pending;  // requests with scans not yet admitted, in turn order
  int64_t next_request = 1;
  int32_t next_matrix = 1;
  epik2_server_stats stats{};
  std::mutex ctx_mu;  // the context is used by the worker and by add_matrix
  std::atomic<int> ctx_waiters{0};  // add_matrix calls waiting for ctx_mu: the worker lets them in

  void finish_scan(Request* r, int32_t scan, const epik2_best* res, int status) {
    if (res) r->results[(size_t)scan] = *res;
    if (status != EPIK2_OK) {
      r->n_failed++;
      r->status = status;
    }
    r->n_done++;
    if (r->n_done == r->n_scans && r->state == kPending) {
      r->state = kDone;
      r->t_done = Clock::now();
      if (r->cancelled) stats.cancelled++;
      else stats.completed++;
    }
  }

  void run() {
    const double target = opts.batch_work > 0 ? opts.batch_work : 2e13;
    const int32_t max_active = std::min(opts.max_active > 0 ? opts.max_active : 256, 512);  // one batched launch
    const int64_t reserve = opts.hbm_reserve_bytes > 0 ? opts.hbm_reserve_bytes : (int64_t)2 << 30;
    for (;;) {
      std::vector<Item> batch;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !pending.empty(); });
        if (stop) return;
        size_t free_b = 0, total_b = 0;
        {
          std::lock_guard<std::mutex> g(ctx_mu);
          epik2_mem_info(ctx, &free_b, &total_b);
        }
        int64_t budget = (int64_t)free_b - reserve;
        double work = 0.0;
        // one scan per pending request in turn; a request leaves the turn order once all
        // its scans are admitted, and the next round starts after the last request served
        size_t blocked = 0;  // consecutive requests whose next scan does not fit now
        while (!pending.empty() && (int32_t)batch.size() < max_active && work < target &&
               blocked < pending.size()) {
          Request* r = pending.front();
          pending.pop_front();
          const int32_t scan = r->n_admitted;
          if (r->cancelled) {  // finish every scan not yet launched
            for (int32_t k = scan; k < r->n_scans; k++) {
              stats.scans_queued--;
              finish_scan(r, k, nullptr, EPIK2_E_CANCELLED);
            }
            r->n_admitted = r->n_scans;
            continue;
          }
          const int64_t bytes = r->dataset >= 0 ? epik2_replicate_bytes(r->n_samples, r->n_snps)
                                                : epik2_dataset_bytes(r->n_samples, r->n_snps);
          if (bytes > (int64_t)total_b - reserve) {  // can never fit: refuse the request's scans
            for (int32_t k = scan; k < r->n_scans; k++) {
              stats.scans_queued--;
              finish_scan(r, k, nullptr, EPIK2_E_NOMEM);
            }
            r->n_admitted = r->n_scans;
            continue;
          }
          if (bytes > budget) {  // admitted once a launch frees memory
            pending.push_back(r);
            blocked++;
            continue;
          }
          blocked = 0;
          budget -= bytes;
          r->n_admitted++;
          stats.scans_queued--;
          batch.push_back(Item{r, scan});
          work += work_of(r->n_samples, r->n_snps);
          if (r->n_admitted < r->n_scans) pending.push_back(r);
        }
        stats.scans_active = (int64_t)batch.size();
        stats.max_active = std::max(stats.max_active, stats.scans_active);
      }
      if (batch.empty()) {  // queued scans wait for device memory held elsewhere
        std::unique_lock<std::mutex> lk(mu);
        cv.wait_for(lk, std::chrono::milliseconds(10));
        continue;
      }
      const auto t0 = Clock::now();
      std::vector<int32_t> ids;
      std::vector<size_t> ok_items;
      std::vector<int> status(batch.size(), EPIK2_OK);
      std::vector<epik2_best> res;
      std::vector<epik2_best> rep_res(batch.size());
      std::vector<char> in_rep(batch.size(), 0);  // scanned in the replicate form
      double kernel_s = 0.0;                       // device time of this launch's search kernels
      int64_t rep_scans = 0;
      for (int spin = 0; spin < 1000 && ctx_waiters.load() > 0; spin++)  // let add_matrix in first
        std::this_thread::sleep_for(std::chrono::microseconds(100));
      {
        std::lock_guard<std::mutex> g(ctx_mu);
        // replicate scans of one resident matrix run in the replicate form (each tile's
        // all-sample counts shared by the replicates) when this launch holds three or more of
        // them: below that the all-sample pass costs about what it saves
        std::map<int32_t, std::vector<size_t>> by_matrix;
        for (size_t b = 0; b < batch.size(); b++)
          if (batch[b].req->dataset >= 0) by_matrix[batch[b].req->dataset].push_back(b);
        for (auto& kv : by_matrix) {
          if (kv.second.size() < 3 || batch[kv.second[0]].req->n_samples >= (1 << 24)) continue;
          const size_t s_n = (size_t)batch[kv.second[0]].req->n_samples;
          std::vector<uint8_t> ph(kv.second.size() * s_n);
          for (size_t t = 0; t < kv.second.size(); t++) {
            const Item& it = batch[kv.second[t]];
            std::memcpy(ph.data() + t * s_n, it.req->phenos.data() + (size_t)it.scan * s_n, s_n);
          }
          std::vector<epik2_best> out(kv.second.size());
          epik2_opts o{};
          o.rescore_fp64 = opts.rescore_fp64;
          const int st = epik2_scan_replicates(ctx, kv.first, ph.data(), (int32_t)kv.second.size(), &o, out.data());
          if (st == EPIK2_OK) {
            epik2_stats cs{};
            epik2_get_stats(ctx, &cs);
            kernel_s += cs.last_scan_kernel_ms * 1e-3;
            rep_scans += (int64_t)kv.second.size();
          }
          for (size_t t = 0; t < kv.second.size(); t++) {
            status[kv.second[t]] = st;
            rep_res[kv.second[t]] = out[t];
            in_rep[kv.second[t]] = 1;
          }
        }
        for (size_t b = 0; b < batch.size(); b++) {
          if (in_rep[b]) continue;
          Request* r = batch[b].req;
          const uint8_t* ph = r->phenos.data() + (size_t)batch[b].scan * (size_t)r->n_samples;
          int32_t id = -1;
          int st = r->dataset >= 0 ? epik2_load_replicate(ctx, r->dataset, ph, &id)
                                   : epik2_load_u8(ctx, r->geno.data(), ph, r->n_samples, r->n_snps, &id);
          status[b] = st;
          if (st == EPIK2_OK) {
            ids.push_back(id);
            ok_items.push_back(b);
          }
        }
        res.resize(ids.size());
        if (!ids.empty()) {
          epik2_opts o{};
          o.rescore_fp64 = opts.rescore_fp64;
          o.stage_words = opts.stage_words;
          const int st = epik2_scan_batch(ctx, ids.data(), (int32_t)ids.size(), &o, res.data());
          if (st != EPIK2_OK)
            for (size_t t : ok_items) status[t] = st;
          else {
            epik2_stats cs{};
            epik2_get_stats(ctx, &cs);
            kernel_s += cs.last_scan_kernel_ms * 1e-3;
          }
        }
        for (int32_t id : ids) epik2_unload(ctx, id);
      }
      const double dt = std::chrono::duration<double>(Clock::now() - t0).count();
      {
        std::lock_guard<std::mutex> lk(mu);
        stats.launches++;
        stats.busy_seconds += dt;
        stats.kernel_seconds += kernel_s;
        stats.replicate_scans += rep_scans;
        size_t q = 0;
        for (size_t b = 0; b < batch.size(); b++) {
          Request* r = batch[b].req;
          const epik2_best* rb = nullptr;
          if (in_rep[b] && status[b] == EPIK2_OK) rb = &rep_res[b];
          if (q < ok_items.size() && ok_items[q] == b) {
            if (status[b] == EPIK2_OK) rb = &res[q];
            q++;
          }
          if (status[b] == EPIK2_OK) {
            stats.scans_done++;
            stats.triplet_samples += work_of(r->n_samples, r->n_snps);
          }
          finish_scan(r, batch[b].scan, rb, status[b]);
        }
        stats.scans_active = 0;
      }
      cv.notify_all();
    }
  }
};

extern "C" {

int epik2_server_create(epik2_server** out, int device, const epik2_server_opts* opts) {
  if (!out) return EPIK2_E_INVALID;
  *out = nullptr;
  std::unique_ptr<epik2_server> s(new epik2_server());
  if (opts) s->opts = *opts;
  int r = epik2_create(&s->ctx, device);
  if (r != EPIK2_OK) return r;
  s->worker = std::thread([p = s.get()] { p->run(); });
  *out = s.release();
  return EPIK2_OK;
}

void epik2_server_destroy(epik2_server* srv) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv.notify_all();
  if (srv->worker.joinable()) srv->worker.join();
  epik2_destroy(srv->ctx);
  delete srv;
}

int epik2_server_add_matrix(epik2_server* srv, const uint8_t* geno, const uint8_t* pheno, int64_t n_samples,
                            int64_t n_snps, int32_t* matrix_id) {
  if (!srv || !matrix_id) return EPIK2_E_INVALID;
  int32_t id = -1;
  int r;
  srv->ctx_waiters++;
  {
    std::lock_guard<std::mutex> g(srv->ctx_mu);
    srv->ctx_waiters--;
    r = epik2_load_u8(srv->ctx, geno, pheno, n_samples, n_snps, &id);
  }
  if (r != EPIK2_OK) return r;
  std::lock_guard<std::mutex> lk(srv->mu);
  const int32_t mid = srv->next_matrix++;
  srv->matrices[mid] = Matrix{id, n_samples, n_snps};
  *matrix_id = mid;
  return EPIK2_OK;
}

static int submit(epik2_server* srv, std::unique_ptr<Request> r, int64_t* request_id) {
  std::lock_guard<std::mutex> lk(srv->mu);
  const int32_t max_q = srv->opts.max_queued > 0 ? srv->opts.max_queued : (1 << 20);
  srv->stats.submitted++;
  if (srv->stats.scans_queued + r->n_scans > max_q) {
    srv->stats.rejected++;
    return EPIK2_E_BUSY;
  }
  r->id = srv->next_request++;
  r->t_submit = Clock::now();
  r->results.assign((size_t)r->n_scans, epik2_best{});
  Request* raw = r.get();
  srv->pending.push_back(raw);
  srv->stats.scans_queued += r->n_scans;
  *request_id = raw->id;
  srv->requests[raw->id] = std::move(r);
  srv->cv.notify_all();
  return EPIK2_OK;
}

int epik2_server_submit_replicates(epik2_server* srv, int32_t matrix_id, const uint8_t* phenos, int32_t n_replicates,
                                   int64_t* request_id) {
  if (!srv || !phenos || !request_id || n_replicates < 1) return EPIK2_E_INVALID;
  std::unique_ptr<Request> r(new Request());
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->matrices.find(matrix_id);
    if (it == srv->matrices.end()) return EPIK2_E_NOT_FOUND;
    r->dataset = it->second.dataset;
    r->n_samples = it->second.n_samples;
    r->n_snps = it->second.n_snps;
  }
  r->n_scans = n_replicates;
  r->phenos.assign(phenos, phenos + (size_t)n_replicates * (size_t)r->n_samples);
  return submit(srv, std::move(r), request_id);
}

int epik2_server_submit_scan(epik2_server* srv, const uint8_t* geno, const uint8_t* pheno, int64_t n_samples,
                             int64_t n_snps, int64_t* request_id) {
  if (!srv || !geno || !pheno || !request_id || n_samples < 1 || n_snps < 3) return EPIK2_E_INVALID;
  std::unique_ptr<Request> r(new Request());
  r->n_samples = n_samples;
  r->n_snps = n_snps;
  r->n_scans = 1;
  r->geno.assign(geno, geno + (size_t)(n_samples * n_snps));
  r->phenos.assign(pheno, pheno + (size_t)n_samples);
  return submit(srv, std::move(r), request_id);
}

int epik2_server_poll(epik2_server* srv, int64_t request_id, epik2_best* out, int32_t capacity, int32_t* n_out,
                      double* latency_seconds) {
  if (!srv) return EPIK2_E_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->requests.find(request_id);
  if (it == srv->requests.end()) return EPIK2_E_NOT_FOUND;
  Request* r = it->second.get();
  if (r->state != kDone) return EPIK2_E_BUSY;
  const int32_t n = out ? std::min(capacity, r->n_scans) : 0;
  for (int32_t k = 0; k < n; k++) out[k] = r->results[(size_t)k];
  if (n_out) *n_out = n;
  if (latency_seconds) *latency_seconds = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  const int status = r->cancelled ? EPIK2_E_CANCELLED : r->status;
  srv->requests.erase(it);
  return status;
}

int epik2_server_cancel(epik2_server* srv, int64_t request_id) {
  if (!srv) return EPIK2_E_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->requests.find(request_id);
  if (it == srv->requests.end()) return EPIK2_E_NOT_FOUND;
  it->second->cancelled = true;
  return EPIK2_OK;
}

int epik2_server_get_stats(epik2_server* srv, epik2_server_stats* out) {
  if (!srv || !out) return EPIK2_E_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  *out = srv->stats;
  return EPIK2_OK;
}

}  // extern "C"
