// server.cu -- continuous-batching query server over one resident index (the
// serving form; the reference answers one query call at a time, lib.rs:775-874).
//
// Clients submit requests (nq query rows, k, epsilon) from any thread; a
// dispatcher thread packs pending queries -- from many requests, of mixed k --
// into device batches of at most `max_batch_queries`, keeps up to
// `max_inflight` batches on the device at once (one stream, pinned staging and
// device buffers per slot, allocated at creation), and admits new queries into
// a slot as soon as its previous batch completes, so requests that arrive while
// others run overlap with them on the device.  Every query carries its own
// parameters (result width, k, rerank width, epsilon, random stream, output
// offset: QueryMeta), and its random stream is its index within its request,
// so each result is identical to the same request run alone through
// rinnd_query / rinnd_query_quantized.  Latency = completion - submission,
// recorded per request by the dispatcher.
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

#include "../../include/rinnd.h"
#include "engine.h"
#include "server.h"

namespace rinnd {
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T>
struct Pinned {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    n = count;
    RINND_CUDA(cudaMallocHost(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T)));
  }
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

struct Request {
  int64_t id = 0;
  int32_t nq = 0, k = 0;
  float eps = 0.f;
  std::vector<float> q;  // nq x D
  std::vector<int32_t> idx;
  std::vector<float> dist;
  int32_t dispatched = 0, completed = 0;
  double t_submit = 0, t_done = 0;
};

struct Chunk {
  std::shared_ptr<Request> req;
  int32_t q0 = 0, nq = 0;
  int64_t out0 = 0;  // offset of the chunk's first output entry in the slot's output
};

struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<Chunk> chunks;
  Pinned<float> hq;
  Pinned<int32_t> hwidth, hkout, hrerank, hidx;
  Pinned<float> heps, hdist;
  Pinned<uint64_t> hstream;
  Pinned<int64_t> hoff;
  DVec<float> dq, dqs;
  DVec<int8_t> dq8;
  DVec<int32_t> dwidth, dkout, drerank, didx;
  DVec<float> deps, ddist;
  DVec<uint64_t> dstream;
  DVec<int64_t> doff;
};

}  // namespace

struct Server {
  ServerIndexView view;
  rinnd_server_params p{};
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> pending;  // not yet fully dispatched
  std::unordered_map<int64_t, std::shared_ptr<Request>> live;
  int64_t next_id = 1, pending_queries = 0;
  bool stop = false;
  std::string error;  // dispatcher failure (sticky)
  // statistics
  std::vector<double> latencies_ms;
  uint64_t batches = 0, batched_queries = 0, completed_requests = 0, completed_queries = 0;
  int32_t peak_inflight = 0;
  std::thread worker;

  void run();
  bool launch(Slot& s);  // packs and launches one batch; false if nothing pending
  void retire(Slot& s);
};

void Server::retire(Slot& s) {
  const double t = now_s();
  std::lock_guard<std::mutex> lock(mu);
  for (const Chunk& c : s.chunks) {
    Request& r = *c.req;
    const size_t n = (size_t)c.nq * (size_t)r.k;
    std::memcpy(r.idx.data() + (size_t)c.q0 * r.k, s.hidx.p + c.out0, n * sizeof(int32_t));
    std::memcpy(r.dist.data() + (size_t)c.q0 * r.k, s.hdist.p + c.out0, n * sizeof(float));
    r.completed += c.nq;
    if (r.completed == r.nq) {
      r.t_done = t;
      latencies_ms.push_back(1000.0 * (r.t_done - r.t_submit));
      ++completed_requests;
      completed_queries += (uint64_t)r.nq;
    }
  }
  s.chunks.clear();
  s.busy = false;
  cv_done.notify_all();
}

bool Server::launch(Slot& s) {
  const int D = view.D, Dp = view.Dp, B = p.max_batch_queries;
  int32_t nq = 0, max_width = 1;
  int64_t out = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    while (!pending.empty() && nq < B) {
      std::shared_ptr<Request> r = pending.front();
      const int32_t take = std::min(r->nq - r->dispatched, B - nq);
      const int32_t width = view.quantized ? quantized_width(r->k, p.candidate_width, p.rerank_width) : r->k;
      const int32_t rr = view.quantized && quantized_rerank(r->k, p.candidate_width, p.rerank_width) ? p.rerank_width : 0;
      for (int32_t t = 0; t < take; ++t) {
        const int32_t qi = r->dispatched + t;
        std::memcpy(s.hq.p + (size_t)(nq + t) * D, r->q.data() + (size_t)qi * D, (size_t)D * sizeof(float));
        s.hwidth.p[nq + t] = width;
        s.hkout.p[nq + t] = r->k;
        s.hrerank.p[nq + t] = rr;
        s.heps.p[nq + t] = r->eps;
        s.hstream.p[nq + t] = (uint64_t)qi;  // the query's index within its request, as when run alone
        s.hoff.p[nq + t] = out + (int64_t)t * r->k;
      }
      s.chunks.push_back(Chunk{r, r->dispatched, take, out});
      out += (int64_t)take * r->k;
      max_width = std::max(max_width, width);
      nq += take;
      r->dispatched += take;
      pending_queries -= take;
      if (r->dispatched == r->nq) pending.pop_front();
    }
  }
  if (nq == 0) return false;
  cudaStream_t st = s.st;
  RINND_CUDA(cudaMemcpy2DAsync(s.dq.p, (size_t)Dp * sizeof(float), s.hq.p, (size_t)D * sizeof(float),
                               (size_t)D * sizeof(float), (size_t)nq, cudaMemcpyHostToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.dwidth.p, s.hwidth.p, nq * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.dkout.p, s.hkout.p, nq * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.drerank.p, s.hrerank.p, nq * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.deps.p, s.heps.p, nq * sizeof(float), cudaMemcpyHostToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.dstream.p, s.hstream.p, nq * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.doff.p, s.hoff.p, nq * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  if (view.normalize) normalize_rows(s.dq.p, nq, D, Dp, st);
  QueryMeta meta;
  meta.width = s.dwidth.p;
  meta.kout = s.dkout.p;
  meta.rerank = s.drerank.p;
  meta.eps = s.deps.p;
  meta.stream = s.dstream.p;
  meta.out_off = s.doff.p;
  if (view.quantized) {
    quantize_rows(s.dq.p, nq, D, Dp, view.index.Dq, view.encoding, view.global_mult, view.index.dim_scales, s.dq8.p,
                  s.dqs.p, st);
    greedy_search_packed(view.index, s.dq.p, s.dq8.p, s.dqs.p, nq, max_width, meta, s.didx.p, s.ddist.p, st,
                         view.stats);
  } else {
    greedy_search_packed(view.index, s.dq.p, nullptr, nullptr, nq, max_width, meta, s.didx.p, s.ddist.p, st,
                         view.stats);
  }
  RINND_CUDA(cudaMemcpyAsync(s.hidx.p, s.didx.p, (size_t)out * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaMemcpyAsync(s.hdist.p, s.ddist.p, (size_t)out * sizeof(float), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaEventRecord(s.done, st));
  s.busy = true;
  std::lock_guard<std::mutex> lock(mu);
  ++batches;
  batched_queries += (uint64_t)nq;
  return true;
}

void Server::run() {
  try {
    RINND_CUDA(cudaSetDevice(view.device));
    for (;;) {
      bool any_busy = false, progressed = false;
      for (auto& sp : slots) {
        Slot& s = *sp;
        if (s.busy) {
          const cudaError_t e = cudaEventQuery(s.done);
          if (e == cudaSuccess) {
            retire(s);
            progressed = true;
          } else if (e != cudaErrorNotReady) {
            RINND_CUDA(e);
          }
        }
        if (!s.busy && launch(s)) progressed = true;
        any_busy |= s.busy;
      }
      int32_t inflight = 0;
      for (auto& sp : slots) inflight += sp->busy ? 1 : 0;
      std::unique_lock<std::mutex> lock(mu);
      peak_inflight = std::max(peak_inflight, inflight);
      if (stop && !any_busy && pending.empty()) return;
      if (!any_busy && pending.empty()) {
        cv_work.wait_for(lock, std::chrono::milliseconds(50));
      } else if (!progressed) {
        lock.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      }
    }
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> lock(mu);
    error = std::string("server dispatcher failed: ") + e.what();
    cv_done.notify_all();
  }
}

Server* server_create(const ServerIndexView& view, const rinnd_server_params& prm) {
  std::unique_ptr<Server> s(new Server());
  s->view = view;
  s->p = prm;
  RINND_CUDA(cudaSetDevice(view.device));
  const int B = prm.max_batch_queries, Dp = view.Dp;
  const size_t outcap = (size_t)B * (size_t)prm.max_k;
  for (int i = 0; i < prm.max_inflight; ++i) {
    std::unique_ptr<Slot> sl(new Slot());
    RINND_CUDA(cudaStreamCreateWithFlags(&sl->st, cudaStreamNonBlocking));
    RINND_CUDA(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
    sl->hq.alloc((size_t)B * view.D);
    sl->hwidth.alloc(B);
    sl->hkout.alloc(B);
    sl->hrerank.alloc(B);
    sl->heps.alloc(B);
    sl->hstream.alloc(B);
    sl->hoff.alloc(B);
    sl->hidx.alloc(outcap);
    sl->hdist.alloc(outcap);
    sl->dq.alloc((size_t)B * Dp, sl->st);
    sl->dq.fill_bytes(0);  // padding columns stay zero
    if (view.quantized) {
      sl->dq8.alloc((size_t)B * view.index.Dq, sl->st);
      sl->dqs.alloc(B, sl->st);
    }
    sl->dwidth.alloc(B, sl->st);
    sl->dkout.alloc(B, sl->st);
    sl->drerank.alloc(B, sl->st);
    sl->deps.alloc(B, sl->st);
    sl->dstream.alloc(B, sl->st);
    sl->doff.alloc(B, sl->st);
    sl->didx.alloc(outcap, sl->st);
    sl->ddist.alloc(outcap, sl->st);
    RINND_CUDA(cudaStreamSynchronize(sl->st));
    s->slots.push_back(std::move(sl));
  }
  Server* raw = s.get();
  s->worker = std::thread([raw] { raw->run(); });
  return s.release();
}

void server_destroy(Server* s) {
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->view.device);
  for (auto& sl : s->slots) {
    cudaStreamSynchronize(sl->st);
    // device buffers are released on their stream before it is destroyed
    sl->dq.release(); sl->dqs.release(); sl->dq8.release(); sl->dwidth.release(); sl->dkout.release();
    sl->drerank.release(); sl->deps.release(); sl->dstream.release(); sl->doff.release(); sl->didx.release();
    sl->ddist.release();
    cudaStreamSynchronize(sl->st);
    cudaEventDestroy(sl->done);
    cudaStreamDestroy(sl->st);
  }
  delete s;
}

int64_t server_submit(Server* s, const float* q, int64_t nq, int32_t k, float eps) {
  std::shared_ptr<Request> r(new Request());
  r->nq = (int32_t)nq;
  r->k = k;
  r->eps = eps;
  r->q.assign(q, q + (size_t)nq * s->view.D);
  r->idx.assign((size_t)nq * k, -1);
  r->dist.assign((size_t)nq * k, 0.f);
  std::lock_guard<std::mutex> lock(s->mu);
  if (!s->error.empty()) throw CudaError(s->error);
  if (s->pending_queries + nq > s->p.max_pending_queries)
    throw ServerBusy("server queue is full (max_pending_queries); poll completed requests and retry");
  r->id = s->next_id++;
  r->t_submit = now_s();
  s->pending.push_back(r);
  s->live[r->id] = r;
  s->pending_queries += nq;
  s->cv_work.notify_all();
  return r->id;
}

bool server_poll(Server* s, int64_t id, int32_t wait_ms, int32_t* out_idx, float* out_dist) {
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) throw std::invalid_argument("unknown or already collected request id");
  std::shared_ptr<Request> r = it->second;
  auto ready = [&] { return r->completed == r->nq || !s->error.empty(); };
  if (!ready() && wait_ms > 0) s->cv_done.wait_for(lock, std::chrono::milliseconds(wait_ms), ready);
  if (!s->error.empty()) throw CudaError(s->error);
  if (r->completed != r->nq) return false;
  if (out_idx) std::memcpy(out_idx, r->idx.data(), r->idx.size() * sizeof(int32_t));
  if (out_dist) std::memcpy(out_dist, r->dist.data(), r->dist.size() * sizeof(float));
  s->live.erase(it);
  return true;
}

const rinnd_server_params& server_params(const Server* s) { return s->p; }

void server_stats(Server* s, rinnd_server_stats* out) {
  std::lock_guard<std::mutex> lock(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed_requests = s->completed_requests;
  out->completed_queries = s->completed_queries;
  out->batches = s->batches;
  out->mean_batch_queries = s->batches ? (double)s->batched_queries / (double)s->batches : 0.0;
  out->peak_inflight = s->peak_inflight;
  out->pending_queries = s->pending_queries;
  if (!s->latencies_ms.empty()) {
    std::vector<double> v = s->latencies_ms;
    auto pct = [&](double f) {
      const size_t i = std::min(v.size() - 1, (size_t)(f * (double)(v.size() - 1) + 0.5));
      std::nth_element(v.begin(), v.begin() + (long)i, v.end());
      return v[i];
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = *std::max_element(v.begin(), v.end());
  }
}

}  // namespace rinnd
