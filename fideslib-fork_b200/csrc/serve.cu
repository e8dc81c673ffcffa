// Continuous-batching request loop over resident evaluation keys.
//
// The reference runs one issuing host thread per context and lets independent host threads
// share it through per-thread scratch slots (FIDESLIB_CONCURRENT_OPS, api/ConcurrentOps.hpp:
// 30-64; test/ConcurrentOpsTests.cu:246-420 checks each lane against its serial result).
// Here a scheduler thread owns the GPU side instead:
//   * submit() only enqueues (thread-safe, non-blocking);
//   * the scheduler forms a batch from the oldest pending request's operation type, taking
//     further requests of that type in arrival order while the batch is below max_batch and
//     the scratch they need fits the HBM budget still free;
//   * each batch is ONE batched launch sequence (op_hmult_batch / op_rotate_batch, any mix
//     of levels) on one of n_streams streams, so batches that are admitted while others are
//     still on the GPU overlap with them;
//   * a host function enqueued behind each batch marks its requests complete (latency =
//     completion - arrival) and returns their budget, waking the scheduler;
//   * bootstrap requests go to registered bootstrap engines (a captured CUDA graph over
//     static buffers, each on its own stream): copy in, graph launch, copy out, so they
//     overlap the HMult / HRotate batches; their memory is the graph's, already resident.
// Results are exact integer arithmetic, so a request's output does not depend on what it
// was batched with; tests/test_serving.py checks that bit for bit.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fides_b200.h"
#include "capi_internal.hpp"
#include "ops.hpp"

namespace fides {
namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  fides_request r;
  uint64_t ticket;
  Clock::time_point arrival;
  size_t bytes;
};

struct Done {
  int status = 0;
  double latency_ms = 0;
  bool ready = false;
};

}  // namespace

struct Server {
  fides_ctx* handle;
  Context* c;
  fides_server_config cfg;
  const uint64_t* relin = nullptr;
  std::map<int, const uint64_t*> rot;  // normalised rotation -> key
  std::vector<cudaStream_t> streams;
  struct BootEngine {
    cudaGraphExec_t exec;
    std::vector<const uint64_t*> in0, in1, out0, out1;  // one static slot per ciphertext it holds
    int in_level, out_level;
    cudaStream_t stream;
    bool busy;
    int capacity() const { return (int)in0.size(); }
  };
  std::deque<BootEngine> boot;  // a deque: registering an engine keeps references to the others valid
  std::vector<bool> busy;

  std::mutex mu;
  std::condition_variable cv;     // scheduler wake-up
  std::condition_variable done_cv;
  std::deque<Pending> pending;
  std::unordered_map<uint64_t, Done> done;
  uint64_t next_ticket = 1;
  size_t in_use = 0;
  bool stop = false;
  // batches of one operation type allowed on the device at once (0 = up to n_streams): with 1,
  // requests that arrive while their type's batch runs wait for it and form the next, larger
  // batch (continuous batching under load), while a type with nothing in flight still starts at once
  int max_inflight_per_op = 0;
  std::map<int, int> inflight;  // op -> batches on the device
  fides_server_stats st{};
  std::thread worker;

  size_t request_bytes(const fides_request& r) const {
    const int l = r.level, ext = l + c->K;
    // the scratch of one key switch (ops.cu ks_limbs): INTT copy, digits, the two extended
    // KSK outputs, two conversions and the two rescale tops; HMult and HRotate need no more
    const size_t limbs = (size_t)l + (size_t)c->beta(l) * ext + 2 * (size_t)ext + 2 * (size_t)l + 2;
    (void)r.op;
    return limbs * c->limb_bytes();
  }

  int norm_rot(int k) const {
    const int h = c->N / 2;
    k %= h;
    return k < 0 ? k + h : k;
  }

  struct Batch {
    Server* s;
    int stream;  // index into streams, or -1 - engine for a bootstrap
    std::vector<uint64_t> tickets;
    std::vector<Clock::time_point> arrivals;
    size_t bytes;
    int status;
    int op = -1;
  };

  static void CUDART_CB on_done(void* p) {
    Batch* b = static_cast<Batch*>(p);
    Server* s = b->s;
    const auto now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (size_t i = 0; i < b->tickets.size(); ++i) {
        Done& d = s->done[b->tickets[i]];
        d.status = b->status;
        d.latency_ms = std::chrono::duration<double, std::milli>(now - b->arrivals[i]).count();
        d.ready = true;
        s->st.completed++;
      }
      s->in_use -= b->bytes;
      if (b->stream >= 0) {
        s->busy[b->stream] = false;
        if (b->op >= 0) s->inflight[b->op]--;
      } else {
        s->boot[-1 - b->stream].busy = false;
      }
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
    delete b;
  }

  void fail_locked(const Pending& p, int code) {
    Done& d = done[p.ticket];
    d.status = code;
    d.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - p.arrival).count();
    d.ready = true;
    st.rejected++;
  }

  // Copy in, graph launch, copy out on the engine's stream, then the completion callback.  An
  // engine that holds several ciphertexts takes up to that many requests at once; slots left
  // empty keep their previous (ignored) contents.
  void launch_bootstrap(BootEngine& e, int index, const std::vector<Pending>& ps) {
    auto* b = new Batch{this, -1 - index, {}, {}, 0, FIDES_OK};
    for (const auto& p : ps) {
      b->tickets.push_back(p.ticket);
      b->arrivals.push_back(p.arrival);
    }
    const size_t lb = c->limb_bytes();
    cudaError_t err = cudaSetDevice(c->device);
    for (size_t k = 0; k < ps.size() && err == cudaSuccess; ++k) {
      err = cudaMemcpyAsync(const_cast<uint64_t*>(e.in0[k]), ps[k].r.c0, lb * e.in_level, cudaMemcpyDeviceToDevice,
                            e.stream);
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(const_cast<uint64_t*>(e.in1[k]), ps[k].r.c1, lb * e.in_level,
                              cudaMemcpyDeviceToDevice, e.stream);
    }
    if (err == cudaSuccess) err = cudaGraphLaunch(e.exec, e.stream);
    for (size_t k = 0; k < ps.size() && err == cudaSuccess; ++k) {
      err = cudaMemcpyAsync(ps[k].r.out0, e.out0[k], lb * e.out_level, cudaMemcpyDeviceToDevice, e.stream);
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(ps[k].r.out1, e.out1[k], lb * e.out_level, cudaMemcpyDeviceToDevice, e.stream);
    }
    if (err != cudaSuccess) b->status = FIDES_ERR_CUDA;
    if (cudaLaunchHostFunc(e.stream, on_done, b) != cudaSuccess) {
      b->status = FIDES_ERR_CUDA;
      on_done(b);
    }
  }

  void run() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv.wait(lk, [&] {
        if (stop) return true;
        if (pending.empty()) return false;
        if (std::find(busy.begin(), busy.end(), false) != busy.end()) return true;
        return std::any_of(boot.begin(), boot.end(), [](const BootEngine& e) { return !e.busy; });
      });
      if (stop && pending.empty()) break;
      if (stop) {
        // shutting down: fail what was never started
        while (!pending.empty()) {
          fail_locked(pending.front(), FIDES_ERR_STATE);
          pending.pop_front();
        }
        done_cv.notify_all();
        break;
      }
      // bootstrap requests, oldest first: the idle engine that best fits the queue (the largest
      // whose capacity the queued bootstraps fill, else the smallest), filled from the queue
      bool launched_boot = false;
      for (;;) {
        int queued = 0;
        for (const auto& p : pending) queued += p.r.op == FIDES_OP_BOOTSTRAP;
        if (!queued) break;
        int best = -1;
        for (size_t e = 0; e < boot.size(); ++e) {
          if (boot[e].busy) continue;
          const int cap = boot[e].capacity();
          if (best < 0) {
            best = (int)e;
            continue;
          }
          const int bc = boot[best].capacity();
          const bool fits = cap <= queued, best_fits = bc <= queued;
          if ((fits && (!best_fits || cap > bc)) || (!fits && !best_fits && cap < bc)) best = (int)e;
        }
        if (best < 0) break;
        BootEngine& eng = boot[best];
        std::vector<Pending> take;
        for (auto it = pending.begin(); it != pending.end() && (int)take.size() < eng.capacity();) {
          if (it->r.op == FIDES_OP_BOOTSTRAP) {
            take.push_back(*it);
            it = pending.erase(it);
          } else {
            ++it;
          }
        }
        eng.busy = true;
        st.batches++;
        st.batched_requests += take.size();
        launched_boot = true;
        lk.unlock();
        launch_bootstrap(eng, best, take);
        lk.lock();
      }
      // the oldest request of a type whose batches may still start (in-flight limit)
      const auto first = std::find_if(pending.begin(), pending.end(), [&](const Pending& p) {
        return p.r.op != FIDES_OP_BOOTSTRAP && (max_inflight_per_op <= 0 || inflight[p.r.op] < max_inflight_per_op);
      });
      const auto free_slot = std::find(busy.begin(), busy.end(), false);
      if (first == pending.end() || free_slot == busy.end()) {
        if (!launched_boot) cv.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      const int slot = (int)(free_slot - busy.begin());
      const int op = first->r.op;
      const size_t budget = cfg.hbm_budget_bytes ? cfg.hbm_budget_bytes : SIZE_MAX;
      std::vector<Pending> take;
      size_t bytes = 0;
      for (auto it = first; it != pending.end() && (int)take.size() < cfg.max_batch;) {
        if (it->r.op != op) {
          ++it;
          continue;
        }
        if (it->bytes > budget) {  // can never fit: reject
          fail_locked(*it, FIDES_ERR_OOM);
          it = pending.erase(it);
          continue;
        }
        if (in_use + bytes + it->bytes > budget) break;  // wait for memory to free up
        bytes += it->bytes;
        take.push_back(*it);
        it = pending.erase(it);
      }
      if (take.empty()) {
        done_cv.notify_all();
        if (in_use == 0 && !pending.empty() && pending.front().r.op == op) continue;
        cv.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
      busy[slot] = true;
      inflight[op]++;
      in_use += bytes;
      st.batches++;
      st.batched_requests += take.size();
      st.peak_bytes = std::max<uint64_t>(st.peak_bytes, in_use);
      lk.unlock();
      auto* b = new Batch{this, slot, {}, {}, bytes, FIDES_OK, op};
      for (auto& p : take) {
        b->tickets.push_back(p.ticket);
        b->arrivals.push_back(p.arrival);
      }
      cudaStream_t s = streams[slot];
      try {
        FIDES_CUDA(cudaSetDevice(c->device));
        if (op == FIDES_OP_ROTATE) {
          std::vector<RotateItem> items;
          for (auto& p : take)
            items.push_back(RotateItem{p.r.c0, p.r.c1, p.r.out0, p.r.out1, rot.at(norm_rot(p.r.rotation)), p.r.level,
                                       h_auto_index(c->logN, p.r.rotation)});
          op_rotate_batch(c, items.data(), (int)items.size(), s);
        } else {
          std::vector<HMultItem> items;
          for (auto& p : take)
            items.push_back(HMultItem{p.r.c0, p.r.c1, p.r.d0, p.r.d1, p.r.out0, p.r.out1, p.r.level});
          op_hmult_batch(c, items.data(), (int)items.size(), relin, op == FIDES_OP_HMULT, s);
        }
      } catch (const Error& e) {
        b->status = e.code;
      } catch (const std::exception&) {
        b->status = FIDES_ERR_STATE;
      }
      cudaError_t e = cudaLaunchHostFunc(s, on_done, b);
      if (e != cudaSuccess) {
        b->status = FIDES_ERR_CUDA;
        on_done(b);
      }
      lk.lock();
    }
  }
};

}  // namespace fides

struct fides_server {
  fides::Server* s;
};

namespace {
template <typename F>
int sguard(F&& f) {
  try {
    f();
    return FIDES_OK;
  } catch (const fides::Error& e) {
    fides::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    fides::set_last_error(e.what());
    return FIDES_ERR_STATE;
  }
}
}  // namespace

extern "C" {

int fides_server_create(fides_ctx* ctx, const fides_server_config* cfg, fides_server** out) {
  return sguard([&] {
    if (!ctx || !ctx->c || !cfg || !out) throw fides::Error(FIDES_ERR_ARG, "null argument");
    if (cfg->n_streams < 1 || cfg->n_streams > 16 || cfg->max_batch < 1)
      throw fides::Error(FIDES_ERR_ARG, "need 1 <= n_streams <= 16 and max_batch >= 1");
    auto* s = new fides::Server();
    s->handle = ctx;
    s->c = ctx->c;
    s->cfg = *cfg;
    FIDES_CUDA(cudaSetDevice(s->c->device));
    s->streams.resize(cfg->n_streams);
    s->busy.assign(cfg->n_streams, false);
    for (auto& st : s->streams) FIDES_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    // grow the scratch pool once to the most the server can have in flight (every stream
    // running a full batch of top-level HMults, capped by the budget), so that admitted
    // batches never map new memory inside the scheduling loop
    {
      fides_request top{};
      top.op = FIDES_OP_HMULT;
      top.level = s->c->n_q;
      size_t most = (size_t)cfg->n_streams * cfg->max_batch * s->request_bytes(top);
      if (cfg->hbm_budget_bytes) most = std::min(most, cfg->hbm_budget_bytes);
      size_t free_b = 0, total_b = 0;
      FIDES_CUDA(cudaMemGetInfo(&free_b, &total_b));
      most = std::min(most, free_b / 2);
      fides::reserve_scratch(s->c, most);
    }
    s->worker = std::thread([s] { s->run(); });
    *out = new fides_server{s};
  });
}

int fides_server_set_relin_key(fides_server* sv, const uint64_t* key) {
  return sguard([&] {
    if (!sv || !key) throw fides::Error(FIDES_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sv->s->mu);
    sv->s->relin = key;
  });
}

int fides_server_add_rotation_key(fides_server* sv, int rotation, const uint64_t* key) {
  return sguard([&] {
    if (!sv || !key) throw fides::Error(FIDES_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sv->s->mu);
    sv->s->rot[sv->s->norm_rot(rotation)] = key;
  });
}

int fides_server_add_bootstrap(fides_server* sv, void* graph_exec, const uint64_t* in0, const uint64_t* in1,
                               int in_level, const uint64_t* out0, const uint64_t* out1, int out_level) {
  return fides_server_add_bootstrap_batch(sv, graph_exec, 1, &in0, &in1, in_level, &out0, &out1, out_level);
}

int fides_server_add_bootstrap_batch(fides_server* sv, void* graph_exec, int capacity, const uint64_t* const* in0,
                                     const uint64_t* const* in1, int in_level, const uint64_t* const* out0,
                                     const uint64_t* const* out1, int out_level) {
  return sguard([&] {
    if (!sv || !graph_exec || !in0 || !in1 || !out0 || !out1) throw fides::Error(FIDES_ERR_ARG, "null argument");
    if (capacity < 1 || capacity > 64) throw fides::Error(FIDES_ERR_ARG, "engine capacity must be 1..64");
    fides::Server* s = sv->s;
    if (in_level < 1 || in_level > s->c->n_q || out_level < 1 || out_level > s->c->n_q)
      throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    fides::Server::BootEngine e{static_cast<cudaGraphExec_t>(graph_exec), {}, {}, {}, {}, in_level, out_level,
                                nullptr, false};
    for (int k = 0; k < capacity; ++k) {
      if (!in0[k] || !in1[k] || !out0[k] || !out1[k]) throw fides::Error(FIDES_ERR_ARG, "null engine buffer");
      e.in0.push_back(in0[k]);
      e.in1.push_back(in1[k]);
      e.out0.push_back(out0[k]);
      e.out1.push_back(out1[k]);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->boot.empty() && (s->boot[0].in_level != in_level || s->boot[0].out_level != out_level))
      throw fides::Error(FIDES_ERR_ARG, "bootstrap engines must share their levels");
    FIDES_CUDA(cudaSetDevice(s->c->device));
    FIDES_CUDA(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
    s->boot.push_back(e);
  });
}

int fides_server_set_max_inflight(fides_server* sv, int max_inflight_per_op) {
  return sguard([&] {
    if (!sv) throw fides::Error(FIDES_ERR_ARG, "null server");
    if (max_inflight_per_op < 0) throw fides::Error(FIDES_ERR_ARG, "negative limit");
    std::lock_guard<std::mutex> lk(sv->s->mu);
    sv->s->max_inflight_per_op = max_inflight_per_op;
  });
}

int fides_server_submit(fides_server* sv, const fides_request* r, uint64_t* ticket) {
  return sguard([&] {
    if (!sv || !r || !ticket) throw fides::Error(FIDES_ERR_ARG, "null argument");
    fides::Server* s = sv->s;
    if (r->level < 1 || r->level > s->c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (!r->c0 || !r->c1 || !r->out0 || !r->out1) throw fides::Error(FIDES_ERR_ARG, "null operand");
    if (r->op == FIDES_OP_ROTATE) {
      std::lock_guard<std::mutex> lk(s->mu);
      if (!s->rot.count(s->norm_rot(r->rotation))) throw fides::Error(FIDES_ERR_KEY, "no key for this rotation");
    } else if (r->op == FIDES_OP_BOOTSTRAP) {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->boot.empty()) throw fides::Error(FIDES_ERR_KEY, "no bootstrap engine registered");
      if (r->level != s->boot[0].in_level) throw fides::Error(FIDES_ERR_LEVEL, "bootstrap input level mismatch");
    } else if (r->op == FIDES_OP_HMULT || r->op == FIDES_OP_HMULT_NORESCALE) {
      if (!r->d0 || !r->d1) throw fides::Error(FIDES_ERR_ARG, "null second operand");
      if (r->op == FIDES_OP_HMULT && r->level < 2) throw fides::Error(FIDES_ERR_LEVEL, "rescale needs level >= 2");
      std::lock_guard<std::mutex> lk(s->mu);
      if (!s->relin) throw fides::Error(FIDES_ERR_KEY, "no relinearization key");
    } else {
      throw fides::Error(FIDES_ERR_ARG, "unknown operation");
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stop) throw fides::Error(FIDES_ERR_STATE, "server is stopping");
      fides::Pending p{*r, s->next_ticket++, fides::Clock::now(), s->request_bytes(*r)};
      *ticket = p.ticket;
      s->done[p.ticket] = fides::Done{};
      s->pending.push_back(p);
      s->st.submitted++;
    }
    s->cv.notify_all();
  });
}

int fides_server_wait(fides_server* sv, uint64_t ticket, double* latency_ms, int* status) {
  return fides_server_wait_timeout(sv, ticket, -1.0, latency_ms, status);
}

int fides_server_wait_timeout(fides_server* sv, uint64_t ticket, double timeout_ms, double* latency_ms,
                              int* status) {
  return sguard([&] {
    if (!sv) throw fides::Error(FIDES_ERR_ARG, "null server");
    fides::Server* s = sv->s;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->done.find(ticket);
    if (it == s->done.end()) throw fides::Error(FIDES_ERR_ARG, "unknown ticket");
    auto ready = [&] { return s->done[ticket].ready; };
    if (timeout_ms < 0) {
      s->done_cv.wait(lk, ready);
    } else if (!s->done_cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
      throw fides::Error(FIDES_ERR_TIMEOUT, "request not complete within the timeout (the ticket stays valid)");
    }
    fides::Done d = s->done[ticket];
    s->done.erase(ticket);
    if (latency_ms) *latency_ms = d.latency_ms;
    if (status) *status = d.status;
  });
}

int fides_server_get_stats(fides_server* sv, fides_server_stats* out) {
  return sguard([&] {
    if (!sv || !out) throw fides::Error(FIDES_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sv->s->mu);
    *out = sv->s->st;
  });
}

int fides_server_destroy(fides_server* sv) {
  return sguard([&] {
    if (!sv) return;
    fides::Server* s = sv->s;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto st : s->streams) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    for (auto& e : s->boot) {
      cudaStreamSynchronize(e.stream);
      cudaStreamDestroy(e.stream);
    }
    delete s;
    delete sv;
  });
}

}  // extern "C"
