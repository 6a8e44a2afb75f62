// server.h -- continuous-batching query server (server.cu) behind rinnd_server_*.
#pragma once
#include <stdexcept>

#include "../../include/rinnd.h"
#include "engine.h"

namespace rinnd {

// What the server needs of an index (the index must outlive the server).
struct ServerIndexView {
  SearchIndex index;
  int device = 0, D = 0, Dp = 0;
  bool normalize = false;
  bool quantized = false;
  int encoding = -1;
  float global_mult = 0.f;
  unsigned long long* stats = nullptr;
};

// Raised when the pending queue is full (RINND_ERR_BUSY).
struct ServerBusy : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// core/index.rs:55-89: result-list width and whether the leading results are reranked.
inline int quantized_width(int k, int candidate_width, int rerank_width) {
  return candidate_width == 0 ? (k > rerank_width ? k : rerank_width) : candidate_width;
}
inline bool quantized_rerank(int k, int candidate_width, int rerank_width) {
  return candidate_width == 0 ? rerank_width > k : rerank_width > 0;
}

struct Server;
Server* server_create(const ServerIndexView& view, const rinnd_server_params& p);
void server_destroy(Server* s);
int64_t server_submit(Server* s, const float* q, int64_t nq, int32_t k, float eps);
// true when the request completed (results copied and the request released)
bool server_poll(Server* s, int64_t id, int32_t wait_ms, int32_t* out_idx, float* out_dist);
void server_stats(Server* s, rinnd_server_stats* out);
const rinnd_server_params& server_params(const Server* s);

}  // namespace rinnd
