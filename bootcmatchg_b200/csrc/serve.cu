// Solve server: continuous batching of solve requests on one GPU.
//
// The reference solves one system per solve() call and keeps no state
// between calls; this is the request loop a serving deployment puts around
// it.  Requests (a matrix identified by a key, one right-hand side) enter a
// FIFO queue and are run by `slots` worker threads, each with its own CUDA
// stream, so the kernels of different solves overlap on the device.
//
//   admission  a request is started when a slot is free and the estimated
//              device footprint of everything resident (cached hierarchies,
//              hierarchies being built, batch work blocks) plus its own stays
//              under mem_cap; idle cached hierarchies are evicted
//              least-recently-used to make room.  A request that does not
//              fit waits; cache hits that need no new memory may pass it.
//   cache      finished hierarchies stay resident keyed by the matrix key
//              (up to cache_cap bytes), so a repeated matrix skips setup.
//   batching   when a worker takes a request, the queued requests with the
//              same key (up to max_batch, in arrival order) join it and run
//              as one multi-right-hand-side solve on the shared hierarchy.
//
// A hierarchy is used by one worker at a time; its solves are deterministic,
// so a request gives the same bits whatever else is running, and a request
// that ran inside a group matches its single solve to the batched solve's
// tolerance.
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

#include "common.cuh"
#include "handle.h"

namespace bcmg {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0, key = 0;
  bcmg_csr A{};  // caller's host arrays; read only if the key needs a setup
  std::vector<double> b;
  double *x = nullptr;  // caller's host output
  Clock::time_point t_submit, t_start, t_done;
  bcmg_solve_info info{};
  bcmg_status status = BCMG_OK;
  std::string error;
  bool done = false;
  int group = 1;
  bool cache_hit = false;
};

struct Entry {
  bcmg_handle *h = nullptr;
  size_t bytes = 0;  // measured after each run (an estimate while building)
  bool busy = false;
  uint64_t last_use = 0;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Footprint estimates used before a hierarchy exists: the input matrix,
// about 0.5x more for coarse levels, the sliced solve copies (and the FP32
// copies in mixed precision), and ~40 work vectors.
size_t estimate_setup(const bcmg_csr &A, const bcmg_ext &e) {
  const double n = A.n, nnz = A.nnz;
  double b = 1.5 * (12.0 * nnz + 4.0 * n) + 1.2 * 8.0 * nnz;
  if (e.precision == BCMG_PREC_MIXED) b += 1.5 * (4.0 * nnz) + 1.2 * 4.0 * nnz;
  b += 40.0 * 8.0 * n;
  return static_cast<size_t>(b);
}

size_t estimate_batch(int32_t n, int m) {
  int W = 1;
  while (W < m && W < 32) W *= 2;
  return static_cast<size_t>(n) * W * (8 * 8 + 4 * 8);
}

// The matrix key of a key-0 submission: a 64-bit hash of n, nnz and the three
// arrays, computed in the submitting thread.  Words of 8 bytes go four at a
// time into four independent lanes (the round of xxHash64: add the word
// times an odd constant, rotate, multiply), the tail bytes of each array
// into one last word; the lanes and the byte count are folded with the
// splitmix64 finalizer.  The lanes' multiplies do not wait on each other,
// so this runs at memory speed, where a byte-at-a-time hash would take most
// of a second for a 700 MB matrix.
uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

uint64_t fold64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

struct KeyHash {
  static constexpr uint64_t kMul = 0x9e3779b185ebca87ull, kRound = 0xc2b2ae3d27d4eb4full;
  uint64_t lane[4] = {0x243f6a8885a308d3ull, 0x13198a2e03707344ull, 0xa4093822299f31d0ull,
                      0x082efa98ec4e6c89ull};
  uint64_t bytes = 0;
  void round(int l, uint64_t w) { lane[l] = rotl64(lane[l] + w * kMul, 31) * kRound; }
  void add(const void *p, size_t n) {
    const unsigned char *c = static_cast<const unsigned char *>(p);
    size_t i = 0;
    uint64_t w[4];
    for (; i + 32 <= n; i += 32) {
      std::memcpy(w, c + i, 32);
      round(0, w[0]);
      round(1, w[1]);
      round(2, w[2]);
      round(3, w[3]);
    }
    for (; i + 8 <= n; i += 8) {
      std::memcpy(w, c + i, 8);
      round(0, w[0]);
    }
    if (i < n) {
      w[0] = 0;
      std::memcpy(w, c + i, n - i);
      round(1, w[0]);
    }
    bytes += n;
  }
  uint64_t finish() const {
    uint64_t h = fold64(bytes);
    for (uint64_t l : lane) h = fold64(h ^ l);
    return h == 0 ? 1 : h;
  }
};

uint64_t hash_csr(const bcmg_csr &A) {
  KeyHash k;
  k.add(&A.n, sizeof(A.n));
  k.add(&A.nnz, sizeof(A.nnz));
  k.add(A.row, sizeof(int32_t) * (static_cast<size_t>(A.n) + 1));
  k.add(A.col, sizeof(int32_t) * static_cast<size_t>(A.nnz));
  k.add(A.val, sizeof(double) * static_cast<size_t>(A.nnz));
  return k.finish();
}

}  // namespace
}  // namespace bcmg

struct bcmg_server {
  bcmg_server_opts opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<bcmg::Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<bcmg::Request>> tickets;
  std::unordered_map<uint64_t, bcmg::Entry> cache;
  size_t cache_bytes = 0;  // every entry, idle, busy or being built
  size_t work_bytes = 0;   // batch work blocks of running groups
  size_t pending_bytes = 0;  // evicted hierarchies not destroyed yet
  int running = 0;
  uint64_t next_ticket = 1, use_clock = 0;
  bool stop = false;
  std::vector<std::thread> workers;
  std::vector<cudaStream_t> streams;
  bcmg_server_stats st{};
};

namespace bcmg {
namespace {

using Group = std::vector<std::shared_ptr<Request>>;

struct Job {
  Group group;
  uint64_t key = 0;
  bool fresh = false;  // needs a setup
  size_t work = 0;     // batch work bytes reserved
};

// Evicted hierarchies still hold their memory until a worker has destroyed
// them outside the lock, so they count as resident until then.
size_t resident(const bcmg_server *s) {
  return s->cache_bytes + s->work_bytes + s->pending_bytes;
}

// An evicted hierarchy and the bytes it was charged.
using Victims = std::vector<std::pair<bcmg_handle *, size_t>>;

size_t idle_bytes(const bcmg_server *s, uint64_t keep) {
  size_t b = 0;
  for (const auto &kv : s->cache)
    if (!kv.second.busy && kv.first != keep) b += kv.second.bytes;
  return b;
}

// Evicts idle entries (other than `keep`), least recently used first, until
// `need` more bytes fit under `cap` or none is left.  The handles go to
// `victims` to be destroyed outside the lock.
void evict_for(bcmg_server *s, size_t need, size_t cap, uint64_t keep, Victims &victims) {
  while (resident(s) + need > cap) {
    auto best = s->cache.end();
    for (auto it = s->cache.begin(); it != s->cache.end(); ++it) {
      if (it->second.busy || it->first == keep) continue;
      if (best == s->cache.end() || it->second.last_use < best->second.last_use) best = it;
    }
    if (best == s->cache.end()) return;
    s->cache_bytes -= best->second.bytes;
    s->pending_bytes += best->second.bytes;
    victims.emplace_back(best->second.h, best->second.bytes);
    s->cache.erase(best);
    ++s->st.evictions;
  }
}

// Picks the next job under the lock, or returns false.
bool pick(bcmg_server *s, Job *job, Victims &victims) {
  const size_t cap = static_cast<size_t>(s->opt.mem_cap_gb * 1e9);
  bool blocked = false;  // an earlier request is waiting for memory
  for (size_t i = 0; i < s->queue.size(); ++i) {
    const std::shared_ptr<Request> r = s->queue[i];  // a copy: erased below
    auto it = s->cache.find(r->key);
    if (it != s->cache.end() && it->second.busy) continue;  // hierarchy in use
    const bool fresh = it == s->cache.end();
    // Same-key requests in arrival order join the group (one at a time with
    // the K-cycle, which batched solves do not run).
    Group g;
    const bcmg_params &pp = s->opt.params;
    const int max_group = pp.cycle_type == 3 || pp.aggrtype == 1 ? 1 : s->opt.max_batch;
    for (size_t j = i; j < s->queue.size() && static_cast<int>(g.size()) < max_group; ++j)
      if (s->queue[j]->key == r->key) g.push_back(s->queue[j]);
    const size_t work = g.size() > 1 ? estimate_batch(r->b.size(), static_cast<int>(g.size())) : 0;
    const size_t need = (fresh ? estimate_setup(r->A, s->opt.ext) : 0) + work;
    if (need > 0 && blocked) continue;  // no overtaking by requests that need memory
    // Evict only when that makes the request fit.
    if (resident(s) + need > cap && resident(s) - idle_bytes(s, r->key) + need <= cap)
      evict_for(s, need, cap, r->key, victims);
    if (resident(s) + need > cap) {
      if (s->running > 0) {
        blocked = true;
        continue;
      }
      if (need > cap) {
        // Cannot fit even on an empty device: fail the group.
        for (auto &q : g) {
          q->status = BCMG_ERR_ALLOC;
          q->error = "estimated device footprint exceeds the server's memory cap";
          q->done = true;
          q->t_start = q->t_done = Clock::now();
          ++s->st.failed;
        }
        for (auto &q : g) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
        s->cv_done.notify_all();
        return pick(s, job, victims);  // the rest of the queue
      }
      // Nothing runs: make all the room there is and admit (the estimate
      // is only an estimate).
      evict_for(s, need, cap, r->key, victims);
    }
    for (auto &q : g) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
    if (fresh) {
      Entry e;
      e.busy = true;
      e.bytes = need - work;
      s->cache[r->key] = e;
      s->cache_bytes += e.bytes;
    } else {
      it->second.busy = true;
    }
    s->work_bytes += work;
    ++s->running;
    job->group = std::move(g);
    job->key = r->key;
    job->fresh = fresh;
    job->work = work;
    return true;
  }
  return false;
}

// Destroys evicted hierarchies on the calling worker's stream.  A handle
// keeps the stream of the worker that ran it last (its runs end with a
// stream synchronize); freeing on that stream could put the frees inside
// another worker's graph capture on it.
// Called without the lock; takes it to release the victims' bytes once they
// are freed (and wakes the workers that may wait for that room).
void destroy_victims(bcmg_server *s, Victims &victims, cudaStream_t stream) {
  if (victims.empty()) return;
  size_t freed = 0;
  for (auto &v : victims) {
    v.first->stream = stream;
    bcmg_destroy(v.first);
    freed += v.second;
  }
  victims.clear();
  std::lock_guard<std::mutex> lk(s->mu);
  s->pending_bytes -= freed;
  s->cv_work.notify_all();
}

// Runs one job on the worker's stream (no lock held).
void run_job(bcmg_server *s, Job &job, cudaStream_t stream, bcmg_handle **hp) {
  const auto t0 = Clock::now();
  for (auto &q : job.group) {
    q->t_start = t0;
    q->group = static_cast<int>(job.group.size());
    q->cache_hit = !job.fresh;
  }
  bcmg_status st = BCMG_OK;
  if (job.fresh) {
    bcmg_ext e = s->opt.ext;
    e.device = s->opt.device;
    e.stream = stream;
    st = bcmg_setup(&job.group[0]->A, &s->opt.params, &e, hp);
  } else {
    // The previous run on this hierarchy ended with a stream synchronize, so
    // it can move to this worker's stream.
    (*hp)->stream = stream;
  }
  const int m = static_cast<int>(job.group.size());
  if (st == BCMG_OK && m == 1) {
    Request &q = *job.group[0];
    std::fill(q.x, q.x + q.b.size(), 0.0);
    st = bcmg_solve(*hp, q.b.data(), q.x, 0, &q.info);
    q.status = st;
    if (st != BCMG_OK) q.error = bcmg_last_error();
  } else if (st == BCMG_OK) {
    const size_t n = job.group[0]->b.size();
    std::vector<double> B(n * m), X(n * m, 0.0);
    for (int c = 0; c < m; ++c)
      std::memcpy(B.data() + c * n, job.group[c]->b.data(), sizeof(double) * n);
    std::vector<bcmg_solve_info> infos(m);
    st = bcmg_solve_batch(*hp, m, B.data(), static_cast<int64_t>(n), X.data(),
                          static_cast<int64_t>(n), 0, infos.data());
    const std::string err = st == BCMG_OK ? std::string() : bcmg_last_error();
    for (int c = 0; c < m; ++c) {
      Request &q = *job.group[c];
      std::memcpy(q.x, X.data() + c * n, sizeof(double) * n);
      q.info = infos[c];
      // A breakdown is reported by the column that met it only.
      q.status = (st == BCMG_ERR_INDEFINITE && infos[c].converged) ? BCMG_OK : st;
      if (q.status != BCMG_OK) q.error = err;
    }
  } else {
    const std::string err = bcmg_last_error();
    for (auto &q : job.group) {
      q->status = st;
      q->error = err;
    }
  }
}

void worker_main(bcmg_server *s, int slot) {
  cudaSetDevice(s->opt.device);
  cudaStream_t stream = s->streams[slot];
  for (;;) {
    Job job;
    Victims victims;
    bcmg_handle *h = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stop && s->queue.empty()) break;
        if (!s->queue.empty() && pick(s, &job, victims)) break;
        if (!victims.empty()) {
          // Free evicted hierarchies before waiting again.
          lk.unlock();
          destroy_victims(s, victims, stream);
          lk.lock();
          continue;
        }
        s->cv_work.wait(lk);
      }
      if (job.group.empty()) {
        lk.unlock();
        destroy_victims(s, victims, stream);
        return;
      }
      if (!job.fresh) h = s->cache[job.key].h;
    }
    destroy_victims(s, victims, stream);
    run_job(s, job, stream, &h);
    const size_t bytes = h ? handle_bytes(h) : 0;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      const auto now = Clock::now();
      auto it = s->cache.find(job.key);
      Entry &e = it->second;
      s->cache_bytes -= e.bytes;
      s->work_bytes -= job.work;
      --s->running;
      if (h) {
        e.h = h;
        e.bytes = bytes;
        e.busy = false;
        e.last_use = ++s->use_clock;
        s->cache_bytes += bytes;
      } else {
        s->cache.erase(it);  // setup failed
      }
      if (job.fresh) ++s->st.setups;
      if (job.group.size() > 1) ++s->st.batches;
      for (auto &q : job.group) {
        q->t_done = now;
        q->done = true;
        ++s->st.completed;
        if (!job.fresh) ++s->st.cache_hits;
        if (q->status != BCMG_OK) ++s->st.failed;
      }
      s->st.peak_resident_bytes =
          std::max<uint64_t>(s->st.peak_resident_bytes, resident(s));
      // Keep the cache within its budget (idle entries only).
      const size_t ccap = static_cast<size_t>(s->opt.cache_cap_gb * 1e9);
      while (s->cache_bytes > ccap) {
        auto best = s->cache.end();
        for (auto jt = s->cache.begin(); jt != s->cache.end(); ++jt)
          if (!jt->second.busy && (best == s->cache.end() ||
                                   jt->second.last_use < best->second.last_use))
            best = jt;
        if (best == s->cache.end()) break;
        s->cache_bytes -= best->second.bytes;
        s->pending_bytes += best->second.bytes;
        victims.emplace_back(best->second.h, best->second.bytes);
        s->cache.erase(best);
        ++s->st.evictions;
      }
      s->cv_done.notify_all();
      s->cv_work.notify_all();
    }
    destroy_victims(s, victims, stream);
  }
}

}  // namespace
}  // namespace bcmg

using namespace bcmg;

extern "C" {

void bcmg_server_opts_default(bcmg_server_opts *o) {
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->slots = 4;
  o->mem_cap_gb = 150.0;
  o->cache_cap_gb = 60.0;
  o->max_batch = 32;
  bcmg_params_default(&o->params);
  bcmg_ext_default(&o->ext);
}

bcmg_status bcmg_server_create(const bcmg_server_opts *opt, bcmg_server **out) {
  clear_error();
  if (!opt || !out) return set_error(BCMG_ERR_PARAM, "null argument");
  *out = nullptr;
  if (opt->slots < 1 || opt->slots > 64 || opt->max_batch < 1 || opt->max_batch > 32 ||
      opt->mem_cap_gb <= 0 || opt->cache_cap_gb < 0)
    return set_error(BCMG_ERR_PARAM, "bad server options");
  BCMG_TRY(bcmg_params_check(&opt->params));
  auto s = std::make_unique<bcmg_server>();
  s->opt = *opt;
  s->opt.ext.stream = nullptr;
  BCMG_CUDA(cudaSetDevice(opt->device));
  for (int i = 0; i < opt->slots; ++i) {
    cudaStream_t st;
    BCMG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    s->streams.push_back(st);
  }
  bcmg_server *raw = s.release();
  for (int i = 0; i < opt->slots; ++i) raw->workers.emplace_back(worker_main, raw, i);
  *out = raw;
  return BCMG_OK;
}

bcmg_status bcmg_server_submit(bcmg_server *s, const bcmg_csr *A, uint64_t key,
                               const double *b, double *x, uint64_t *ticket) {
  clear_error();
  if (!s || !A || !b || !x || !ticket) return set_error(BCMG_ERR_PARAM, "null argument");
  if (A->n <= 0 || A->n != A->m || !A->row || !A->col || !A->val)
    return set_error(BCMG_ERR_INVALID_MATRIX, "square host CSR matrix required");
  auto r = std::make_shared<Request>();
  r->key = key ? key : hash_csr(*A);
  r->A = *A;
  r->b.assign(b, b + A->n);
  r->x = x;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return set_error(BCMG_ERR_PARAM, "server is shutting down");
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->queue.push_back(r);
    ++s->st.submitted;
  }
  s->cv_work.notify_one();
  *ticket = r->ticket;
  return BCMG_OK;
}

bcmg_status bcmg_server_wait(bcmg_server *s, uint64_t ticket, double timeout_s,
                             bcmg_request_info *info) {
  clear_error();
  if (!s) return set_error(BCMG_ERR_PARAM, "null server");
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return set_error(BCMG_ERR_PARAM, "unknown ticket %llu",
                                                 static_cast<unsigned long long>(ticket));
    r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_s < 0) {
      s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
      return set_error(BCMG_ERR_PENDING, "request %llu still pending",
                       static_cast<unsigned long long>(ticket));
    }
    s->tickets.erase(ticket);
  }
  if (info) {
    info->solve = r->info;
    info->latency_ms = ms_between(r->t_submit, r->t_done);
    info->queue_ms = ms_between(r->t_submit, r->t_start);
    info->group = r->group;
    info->cache_hit = r->cache_hit ? 1 : 0;
  }
  if (r->status != BCMG_OK) return set_error(r->status, "%s", r->error.c_str());
  return BCMG_OK;
}

bcmg_status bcmg_server_stats_get(bcmg_server *s, bcmg_server_stats *out) {
  if (!s || !out) return set_error(BCMG_ERR_PARAM, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident_bytes = resident(s);
  out->cached_hierarchies = static_cast<int>(s->cache.size());
  out->queued = static_cast<int>(s->queue.size());
  out->running = s->running;
  return BCMG_OK;
}

bcmg_status bcmg_server_destroy(bcmg_server *s) {
  if (!s) return BCMG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->workers) t.join();
  cudaSetDevice(s->opt.device);
  for (auto &kv : s->cache)
    if (kv.second.h) bcmg_destroy(kv.second.h);
  for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
  delete s;
  return BCMG_OK;
}

}  // extern "C"
