// Continuous-batching top-k server over a resident reference set (C ABI gpusw_server_*).
// Included at the end of engine.cu: it drives the same planner and kernels.
//
// Threads: callers submit/poll/cancel under `mu`; one scheduler thread owns the slots.
// Each slot is a private context (own CUDA stream and buffers) that borrows the owner's
// resident reference set; a batch is the concatenated queries of the request parts
// admitted together, scored by one planned launch sequence followed by the top-k kernel,
// with the results copied into pinned host memory and an event recorded. The scheduler
// polls the events (no device-side waits anywhere), copies finished parts into their
// requests and admits more work while a slot and the memory budget allow.
//
// Batches are cut by work, not by request: a batch holds about batch_cells cells, and
// while other requests wait no request takes more than half of it, so a large request runs
// as several parts and small requests that arrive behind it share the next batch instead of
// waiting for it to finish (chunked, fair-share continuous batching). Requests are still
// served in arrival order; a request completes when its last part does.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>

#define GPUSW_REQ_FAILED 4

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Default target work per batch (gpusw_server_set_batch_cells changes it).
constexpr double kServeBatchCells = 3e12;

struct SrvRequest {
  int64_t id = 0;
  int nq = 0;
  int next_q = 0;   // queries handed to batches so far
  int parts = 0;    // parts in flight
  bool failed = false;
  std::vector<uint8_t> codes;
  std::vector<int32_t> offsets;  // rebased to 0, nq + 1 entries
  int state = GPUSW_REQ_PENDING;
  bool cancel = false;
  std::vector<int32_t> idx, sc;
  double t_submit = 0, t_done = 0, cells = 0;
  int64_t bytes = 0;  // device bytes the request adds to a batch
  int max_len = 0;
};

struct Slot {
  gpusw_ctx* ctx = nullptr;
  Db q;                          // the batch's query set (storage below, grow-only)
  DevBuf words, woff, len, perm, ident;
  std::vector<uint32_t> hwords;
  struct Part { SrvRequest* r; int q0, nq, row0; };
  std::vector<Part> parts;
  int nq = 0, P = 2;
  int64_t bytes = 0;
  cudaEvent_t done = nullptr;
  int32_t* h_idx = nullptr;      // pinned results
  int32_t* h_sc = nullptr;
  int* h_flag = nullptr;
  size_t h_cap = 0;
  bool busy = false;
};

}  // namespace

struct gpusw_server {
  gpusw_ctx* owner = nullptr;
  Db* refs = nullptr;
  int kk = 0, dtype = 0;
  double ref_residues = 0;  // total length of the resident references
  double batch_cells = kServeBatchCells;
  int64_t budget = 4ll << 30, in_use = 0;
  int max_slots = 2, max_batch = 1024, max_pending = 4096;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  std::deque<SrvRequest*> pending;
  std::unordered_map<int64_t, std::unique_ptr<SrvRequest>> reqs;
  int64_t next_id = 1;
  std::thread worker;
  bool stop = false;
  std::string err, worker_err;
  int64_t submitted = 0, completed = 0, cancelled = 0, rejected = 0, batches = 0, batch_q = 0;
  std::vector<double> lat;
  double cells = 0, t_first = -1;
};

namespace {

int64_t request_bytes(const gpusw_server* s, int nq, int64_t residues) {
  // score block + top-k + packed queries (<= 1 byte per residue) + per-query metadata
  return (int64_t)nq * s->refs->n * 4 + (int64_t)nq * s->kk * 8 + residues + (int64_t)nq * 32;
}

// Pack the batch's queries into the slot's query set (host packing, async upload).
void slot_upload(Slot& sl) {
  gpusw_ctx* c = sl.ctx;
  Db& q = sl.q;
  int n = 0, maxc = 0;
  for (const Slot::Part& pt : sl.parts) n += pt.nq;
  q.n = n;
  q.len.assign(n, 0);
  q.woff.assign(n, 0);
  q.max_len = 0;
  int i = 0;
  for (const Slot::Part& pt : sl.parts) {
    const SrvRequest* r = pt.r;
    for (int a = pt.q0; a < pt.q0 + pt.nq; ++a, ++i) {
      q.len[i] = r->offsets[a + 1] - r->offsets[a];
      q.max_len = std::max(q.max_len, q.len[i]);
      for (int c = r->offsets[a]; c < r->offsets[a + 1]; ++c) maxc = std::max<int>(maxc, r->codes[c]);
    }
  }
  q.max_code = maxc;
  q.bits = maxc < 4 ? 2 : maxc < 16 ? 4 : maxc < 32 ? 5 : 8;
  q.per = q.bits == 5 ? 6 : 32 / q.bits;
  long long w = 0;
  for (int a = 0; a < n; ++a) {
    q.woff[a] = w;
    w += ((q.len[a] + q.per - 1) / q.per + 3) & ~3ll;
  }
  const long long nwords = w + 64;
  sl.hwords.assign((size_t)nwords, 0u);
  i = 0;
  for (const Slot::Part& pt : sl.parts) {
    const SrvRequest* r = pt.r;
    for (int a = pt.q0; a < pt.q0 + pt.nq; ++a, ++i) {
      const uint8_t* src = r->codes.data() + r->offsets[a];
      uint32_t* dst = sl.hwords.data() + q.woff[i];
      for (int cidx = 0; cidx < q.len[i]; cidx += q.per) {
        uint32_t v = 0;
        const int e_end = std::min(q.per, q.len[i] - cidx);
        for (int e = 0; e < e_end; ++e) v |= (uint32_t)src[cidx + e] << (e * q.bits);
        dst[cidx / q.per] = v;
      }
    }
  }
  q.perm_desc.resize(n);
  std::iota(q.perm_desc.begin(), q.perm_desc.end(), 0);
  q.order_ready = true;  // a query set: never used as references
  q.words = sl.words.as<uint32_t>((size_t)nwords);
  q.woff_d = sl.woff.as<long long>((size_t)std::max(1, n));
  q.len_d = sl.len.as<int>((size_t)std::max(1, n));
  q.perm_d = sl.perm.as<int>((size_t)std::max(1, n));
  q.ident_d = sl.ident.as<int>((size_t)std::max(1, n));
  CK(cudaMemcpyAsync(q.words, sl.hwords.data(), nwords * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(q.woff_d, q.woff.data(), n * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(q.len_d, q.len.data(), n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
}

// Enqueue the batch of slot `sl` (scoring, top-k, copies to pinned memory, done event).
void slot_launch(gpusw_server* s, Slot& sl, int P) {
  gpusw_ctx* c = sl.ctx;
  set_device(c);
  sl.P = P;
  const int nq = sl.q.n, nr = s->refs->n, kk = s->kk;
  Bufs& B = c->shared;
  B.reset_marks();
  CK(cudaMemsetAsync(B.ovf_flag.as<int>(1), 0, sizeof(int), c->stream));
  std::vector<int32_t> qlist(nq);
  std::iota(qlist.begin(), qlist.end(), 0);
  int* d_out = B.out.as<int>((size_t)nq * nr);
  int* d_idx = B.idx.as<int>((size_t)nq * kk);
  int* d_sc = B.sc.as<int>((size_t)nq * kk);
  run_cross(c, B, sl.q, *s->refs, qlist.data(), nq, P, d_out, nr);
  launch_topk(d_out, nq, nr, kk, d_idx, d_sc, c->stream);
  CK(cudaGetLastError());
  const size_t need = (size_t)nq * kk;
  if (need > sl.h_cap) {
    if (sl.h_idx) cudaFreeHost(sl.h_idx);
    if (sl.h_sc) cudaFreeHost(sl.h_sc);
    sl.h_idx = sl.h_sc = nullptr;
    sl.h_cap = std::max(need, (size_t)1024);
    CK(cudaMallocHost(&sl.h_idx, sl.h_cap * 4));
    CK(cudaMallocHost(&sl.h_sc, sl.h_cap * 4));
  }
  if (!sl.h_flag) CK(cudaMallocHost(&sl.h_flag, sizeof(int)));
  if (need) {
    CK(cudaMemcpyAsync(sl.h_idx, d_idx, need * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(sl.h_sc, d_sc, need * 4, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaMemcpyAsync(sl.h_flag, B.ovf_flag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(sl.done, c->stream));
}

// Scheduler: finish completed batches, admit pending requests into free slots.
void server_loop(gpusw_server* s) {
  cudaSetDevice(s->owner->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool any_busy = false, progressed = false;
    for (auto& slp : s->slots) {
      Slot& sl = *slp;
      if (!sl.busy) continue;
      if (cudaEventQuery(sl.done) != cudaSuccess) {
        any_busy = true;
        continue;
      }
      std::string fail_msg;
      try {
        if (sl.P == 2 && *sl.h_flag > kOvfCap) {  // rare: rescore the whole batch in int32
          slot_launch(s, sl, 1);
          CK(cudaEventSynchronize(sl.done));
        }
      } catch (const Error& e) {
        fail_msg = e.msg;
      }
      const double t = now_ms();
      const int kk = s->kk;
      for (const Slot::Part& pt : sl.parts) {
        SrvRequest* r = pt.r;
        --r->parts;
        if (!fail_msg.empty()) {
          r->failed = true;
          s->worker_err = fail_msg;
        } else if (!r->cancel && kk > 0) {
          std::copy(sl.h_idx + (size_t)pt.row0 * kk, sl.h_idx + (size_t)(pt.row0 + pt.nq) * kk,
                    r->idx.begin() + (size_t)pt.q0 * kk);
          std::copy(sl.h_sc + (size_t)pt.row0 * kk, sl.h_sc + (size_t)(pt.row0 + pt.nq) * kk,
                    r->sc.begin() + (size_t)pt.q0 * kk);
        }
        if (r->parts > 0 || (r->next_q < r->nq && !r->cancel && !r->failed)) continue;
        // the request's last part is back
        if (r->failed) {
          r->state = GPUSW_REQ_FAILED;
        } else if (r->cancel) {
          r->state = GPUSW_REQ_CANCELLED;
          ++s->cancelled;
        } else {
          r->state = GPUSW_REQ_DONE;
          r->t_done = t;
          s->lat.push_back(t - r->t_submit);
          s->cells += r->cells;
          ++s->completed;
        }
        r->codes.clear();
        r->codes.shrink_to_fit();
      }
      sl.parts.clear();
      sl.busy = false;
      s->in_use -= sl.bytes;
      progressed = true;
    }
    if (progressed) s->done_cv.notify_all();
    // admissions: parts of the pending requests, in arrival order, cut by work
    for (auto& slp : s->slots) {
      Slot& sl = *slp;
      if (sl.busy || s->pending.empty() || s->stop) continue;
      int64_t bytes = 0;
      int nq = 0, max_len = 0;
      double cells = 0;
      std::vector<Slot::Part> take;
      // The batch grows with the backlog: at least batch_cells, and an equal share of the
      // queued work per slot when more is waiting (bigger batches keep the device fuller
      // when requests queue anyway; a short queue keeps batches, and latency, small). With
      // company in the queue no request takes more than half a batch.
      double backlog = 0;
      for (const SrvRequest* r : s->pending)
        backlog += (double)(r->offsets[r->nq] - r->offsets[r->next_q]) * s->ref_residues;
      const double target = std::max(s->batch_cells, backlog / (double)s->slots.size());
      const double share = s->pending.size() > 1 ? target / 2 : target;
      for (size_t qi = 0; qi < s->pending.size() && nq < s->max_batch && cells < target;) {
        SrvRequest* r = s->pending[qi];
        Slot::Part pt{r, r->next_q, 0, nq};
        double rcells = 0;
        int64_t rbytes = 0;
        while (r->next_q < r->nq && nq < s->max_batch) {
          const int a = r->next_q;
          const int len = r->offsets[a + 1] - r->offsets[a];
          const double qc = (double)len * s->ref_residues;
          const int64_t qb = request_bytes(s, 1, len);
          const bool first = take.empty() && pt.nq == 0;
          if (!first && (rcells + qc > share || cells + qc > target)) break;
          if (s->in_use + bytes + rbytes + qb > s->budget) break;
          rcells += qc;
          rbytes += qb;
          ++pt.nq;
          ++nq;
          ++r->next_q;
          max_len = std::max(max_len, len);
        }
        if (pt.nq == 0) break;  // budget or batch full: the rest waits
        cells += rcells;
        bytes += rbytes;
        take.push_back(pt);
        ++r->parts;
        if (r->state == GPUSW_REQ_PENDING) {
          r->state = GPUSW_REQ_RUNNING;
          if (s->kk > 0) {
            r->idx.assign((size_t)r->nq * s->kk, 0);
            r->sc.assign((size_t)r->nq * s->kk, 0);
          }
        }
        if (r->next_q == r->nq) s->pending.erase(s->pending.begin() + (long)qi);
        else ++qi;
      }
      if (take.empty()) break;  // the head request waits for memory to free up
      sl.parts = take;
      sl.bytes = bytes;
      s->in_use += bytes;
      sl.busy = true;
      any_busy = true;
      ++s->batches;
      s->batch_q += nq;
      lk.unlock();
      std::string fail_msg;
      try {
        slot_upload(sl);
        const int P = choose_width(sl.ctx, s->dtype, max_len, s->refs->max_len);
        slot_launch(s, sl, P);
      } catch (const Error& e) {
        fail_msg = e.msg;
      }
      lk.lock();
      if (!fail_msg.empty()) {  // the batch failed before reaching the device
        for (const Slot::Part& pt : sl.parts) {
          pt.r->failed = true;
          s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), pt.r), s->pending.end());
          if (--pt.r->parts == 0) pt.r->state = GPUSW_REQ_FAILED;
        }
        s->worker_err = fail_msg;
        sl.parts.clear();
        sl.busy = false;
        s->in_use -= sl.bytes;
        s->done_cv.notify_all();
      }
    }
    if (s->stop && !any_busy) break;
    if (any_busy) {
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(50));
      lk.lock();
    } else {
      s->work_cv.wait_for(lk, std::chrono::milliseconds(20));
    }
  }
}

}  // namespace

extern "C" {

int gpusw_server_create(gpusw_ctx* ctx, int32_t rdb, int32_t k, int dtype, int64_t mem_budget,
                        int32_t max_slots, int32_t max_batch_queries, int32_t max_pending,
                        gpusw_server** out) {
  if (!out) return GPUSW_ERR_INVALID;
  *out = nullptr;
  auto srv = std::make_unique<gpusw_server>();
  int rc = guarded(ctx, [&] {
    Db& r = get_db(ctx, rdb);
    if (!ctx->has_scheme) fail(GPUSW_ERR_SCHEME, "no scheme set");
    ensure_row_order(ctx, r);
    if (r.max_code >= ctx->sch.ns) fail(GPUSW_ERR_INVALID, "reference codes exceed the scheme's table");
    if (k < 0 || max_slots < 1 || max_slots > 8 || max_batch_queries < 1 || max_pending < 1)
      fail(GPUSW_ERR_INVALID, "bad server limits");
    srv->owner = ctx;
    srv->refs = &r;
    srv->kk = std::min(k, r.n);
    for (int l : r.len) srv->ref_residues += l;
    srv->dtype = dtype;
    if (mem_budget > 0) srv->budget = mem_budget;
    srv->max_slots = max_slots;
    srv->max_batch = max_batch_queries;
    srv->max_pending = max_pending;
    set_device(ctx);
    if (ctx->sch.mode == gsw::kModeLocal && ctx->sch.ns <= 126) get_stream(ctx, r, false);
    ensure_tuned(ctx, 2);
    ensure_tuned(ctx, 1);
    CK(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < max_slots; ++i) {
      auto sl = std::make_unique<Slot>();
      int src = gpusw_ctx_create(ctx->device, &sl->ctx);
      if (src != GPUSW_OK) fail(src, "slot context creation failed");
      const HostScheme& h = ctx->sch;
      src = gpusw_set_scheme(sl->ctx, h.mode, h.go, h.ge, h.free_q, h.free_r, h.ns, h.sub.data());
      if (src != GPUSW_OK) fail(src, gpusw_last_error(sl->ctx));
      for (DevBuf* b : {&sl->words, &sl->woff, &sl->len, &sl->perm, &sl->ident}) b->held = &sl->ctx->held;
      sl->ctx->tune = ctx->tune;
      CK(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
      srv->slots.push_back(std::move(sl));
    }
  });
  if (rc != GPUSW_OK) {
    for (auto& sl : srv->slots) {
      if (sl->done) cudaEventDestroy(sl->done);
      for (DevBuf* b : {&sl->words, &sl->woff, &sl->len, &sl->perm, &sl->ident}) b->release();
      gpusw_ctx_destroy(sl->ctx);
    }
    return rc;
  }
  gpusw_server* s = srv.release();
  s->worker = std::thread(server_loop, s);
  *out = s;
  return GPUSW_OK;
}

int gpusw_server_submit(gpusw_server* s, const uint8_t* codes, const int32_t* offsets, int32_t nq,
                        int64_t* req_id) {
  if (!s || !req_id || !offsets || nq < 0) return GPUSW_ERR_INVALID;
  auto r = std::make_unique<SrvRequest>();
  r->nq = nq;
  const int32_t base = offsets[0];
  if (base < 0) return GPUSW_ERR_INVALID;
  r->offsets.resize(nq + 1);
  double qsum = 0;
  for (int a = 0; a <= nq; ++a) {
    r->offsets[a] = offsets[a] - base;
    if (a > 0) {
      if (r->offsets[a] < r->offsets[a - 1]) {
        std::lock_guard<std::mutex> g(s->mu);
        s->err = "offsets must be non-decreasing";
        return GPUSW_ERR_INVALID;
      }
      const int l = r->offsets[a] - r->offsets[a - 1];
      r->max_len = std::max(r->max_len, l);
      qsum += l;
    }
  }
  const int64_t total = r->offsets[nq];
  if (total > 0 && !codes) return GPUSW_ERR_INVALID;
  r->codes.assign(codes + base, codes + base + total);
  for (uint8_t v : r->codes)
    if (v >= s->owner->sch.ns) {
      std::lock_guard<std::mutex> g(s->mu);
      s->err = "query codes exceed the scheme's table";
      return GPUSW_ERR_INVALID;
    }
  double rsum = 0;
  for (int l : s->refs->len) rsum += l;
  r->cells = qsum * rsum;
  r->bytes = request_bytes(s, nq, total);
  r->t_submit = now_ms();
  std::lock_guard<std::mutex> g(s->mu);
  if (r->bytes > s->budget) {
    ++s->rejected;
    s->err = "request needs more device memory than the server's budget";
    return GPUSW_ERR_MEMORY;
  }
  if ((int)s->pending.size() >= s->max_pending) {
    ++s->rejected;
    s->err = "admission queue full";
    return GPUSW_ERR_QUEUE_FULL;
  }
  if (s->t_first < 0) s->t_first = r->t_submit;
  r->id = s->next_id++;
  *req_id = r->id;
  if (nq == 0) {  // nothing to score
    r->state = GPUSW_REQ_DONE;
    r->t_done = r->t_submit;
    ++s->completed;
    s->lat.push_back(0.0);
  } else {
    s->pending.push_back(r.get());
  }
  s->reqs[r->id] = std::move(r);
  ++s->submitted;
  s->work_cv.notify_one();
  return GPUSW_OK;
}

int gpusw_server_poll(gpusw_server* s, int64_t req_id, int32_t timeout_ms, int32_t* state,
                      int32_t* out_idx, int32_t* out_score) {
  if (!s || !state) return GPUSW_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) {
    s->err = "unknown request id";
    return GPUSW_ERR_NOT_FOUND;
  }
  SrvRequest* r = it->second.get();
  if (timeout_ms > 0 && (r->state == GPUSW_REQ_PENDING || r->state == GPUSW_REQ_RUNNING))
    s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
      return r->state != GPUSW_REQ_PENDING && r->state != GPUSW_REQ_RUNNING;
    });
  *state = r->state;
  if (r->state == GPUSW_REQ_DONE) {
    if (out_idx && !r->idx.empty()) memcpy(out_idx, r->idx.data(), r->idx.size() * 4);
    if (out_score && !r->sc.empty()) memcpy(out_score, r->sc.data(), r->sc.size() * 4);
    s->reqs.erase(it);
    return GPUSW_OK;
  }
  if (r->state == GPUSW_REQ_CANCELLED) {
    s->reqs.erase(it);
    return GPUSW_OK;
  }
  if (r->state == GPUSW_REQ_FAILED) {
    s->err = s->worker_err;
    s->reqs.erase(it);
    return GPUSW_ERR_CUDA;
  }
  return timeout_ms > 0 ? GPUSW_ERR_TIMEOUT : GPUSW_OK;
}

int gpusw_server_cancel(gpusw_server* s, int64_t req_id) {
  if (!s) return GPUSW_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) {
    s->err = "unknown request id";
    return GPUSW_ERR_NOT_FOUND;
  }
  SrvRequest* r = it->second.get();
  if (r->state == GPUSW_REQ_PENDING) {
    s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), r), s->pending.end());
    r->state = GPUSW_REQ_CANCELLED;
    ++s->cancelled;
    s->done_cv.notify_all();
  } else if (r->state == GPUSW_REQ_RUNNING) {
    // parts not yet handed out are dropped; the request ends when its last part is back,
    // or now if none is on the device
    r->cancel = true;
    s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), r), s->pending.end());
    if (r->parts == 0) {
      r->state = GPUSW_REQ_CANCELLED;
      ++s->cancelled;
      r->codes.clear();
      s->done_cv.notify_all();
    }
  }
  return GPUSW_OK;
}

int gpusw_server_get_stats(gpusw_server* s, gpusw_server_stats* out) {
  if (!s || !out) return GPUSW_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  gpusw_server_stats st{};
  st.submitted = s->submitted;
  st.completed = s->completed;
  st.cancelled = s->cancelled;
  st.rejected = s->rejected;
  st.pending = (int64_t)s->pending.size();
  for (auto& sl : s->slots)
    if (sl->busy) st.running += (int64_t)sl->parts.size();
  st.batches = s->batches;
  st.mean_batch_queries = s->batches ? (double)s->batch_q / s->batches : 0.0;
  if (!s->lat.empty()) {
    std::vector<double> v = s->lat;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      const size_t i = (size_t)std::min<double>(v.size() - 1, std::ceil(p * v.size()) - 1);
      return v[i];
    };
    st.p50_ms = pct(0.50);
    st.p99_ms = pct(0.99);
    st.max_ms = v.back();
    st.mean_ms = std::accumulate(v.begin(), v.end(), 0.0) / v.size();
  }
  st.cells = s->cells;
  st.wall_s = s->t_first < 0 ? 0.0 : (now_ms() - s->t_first) * 1e-3;
  st.gcups = st.wall_s > 0 ? s->cells / st.wall_s / 1e9 : 0.0;
  for (auto& sl : s->slots) st.device_bytes += sl->ctx->held;
  *out = st;
  return GPUSW_OK;
}

int gpusw_server_set_batch_cells(gpusw_server* s, double cells) {
  if (!s || cells < 0) return GPUSW_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  s->batch_cells = cells > 0 ? cells : kServeBatchCells;
  return GPUSW_OK;
}

const char* gpusw_server_last_error(const gpusw_server* s) { return s ? s->err.c_str() : ""; }

void gpusw_server_destroy(gpusw_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    for (SrvRequest* r : s->pending) r->state = GPUSW_REQ_CANCELLED;
    s->pending.clear();
  }
  s->work_cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (auto& sl : s->slots) {
    if (sl->done) cudaEventDestroy(sl->done);
    if (sl->h_idx) cudaFreeHost(sl->h_idx);
    if (sl->h_sc) cudaFreeHost(sl->h_sc);
    if (sl->h_flag) cudaFreeHost(sl->h_flag);
    for (DevBuf* b : {&sl->words, &sl->woff, &sl->len, &sl->perm, &sl->ident}) b->release();
    gpusw_ctx_destroy(sl->ctx);
  }
  delete s;
}

}  // extern "C"
