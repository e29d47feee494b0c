// server.cu -- continuous-batching Groth16 prove server (host code).
//
// Replaces the reference's single-proof-at-a-time TCP server loop (src/python/
// groth_prover.py:808-891 startServer, which drops requests that arrive while a proof is
// running and re-copies the proving key to the GPU for every proof).  Here:
//   * proving keys stay resident in HBM (cs_pk, with their fixed-base MSM tables), and the
//     NTT twiddles stay resident in each slot's context;
//   * requests queue FIFO; each of `slots` worker threads owns a context (its own streams
//     and scratch arena) and takes the next request as soon as it is free AND the request
//     is admitted by device memory: free memory (cudaMemGetInfo) minus the bytes promised
//     to admitted requests whose slots have not grown yet must cover the slot's scratch
//     growth plus `reserve`; a slot grows once for every registered key where that fits
//     (else for the request's key), so it does not grow, free and synchronise the device
//     again in steady state; an admitted slot grows its buffers at once and then withdraws
//     its promise, since cudaMemGetInfo counts the memory from then on;
//   * admitted proofs run concurrently on the device: one proof's MSM tails, QAP and
//     H step overlap the next one's bucket accumulation;
//   * a slot that takes a request of a small circuit (up to 2^16 constraints) takes the
//     queued requests with the same key along (up to max_batch, a power of two) and proves
//     them in one cs_prove_batch_device pass: their MSMs share one digit sort and one
//     bucket accumulation, and the pass replays as one CUDA graph.
// Results do not depend on the mix: every proof is computed by the same kernels on its
// own slot scratch (a test compares proofs made alone and in a mix, byte for byte).
#include <algorithm>
#include <atomic>
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

#include "../../include/cusnarks_b200.h"
#include "runtime.cuh"

namespace csb {
size_t prove_workspace_bytes(const cs_pk* pk);
uint32_t pk_n_vars(const cs_pk* pk);
cudaError_t ctx_reserve(cs_ctx* ctx, size_t work_bytes, size_t in_bytes);
uint32_t pk_domain(const cs_pk* pk);
bool pk_has_fixed(const cs_pk* pk);
bool prove_batch_ready(cs_ctx* ctx, const cs_pk* pk, uint32_t k);
}  // namespace csb

namespace {

constexpr size_t kLatRing = 1024;
constexpr uint32_t kMinBatch = 4;  // fewer same-key requests are proved one by one

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
  uint64_t id = 0;
  int key = 0;
  cs_pk* pk = nullptr;
  const uint32_t* w = nullptr;
  uint32_t r[8], s[8];
  uint32_t* proof = nullptr;
  int status = CS_OK;
  bool done = false;
  double t_submit = 0, t_start = 0, t_end = 0;
  float device_ms = 0.f;
  std::string err;
};

}  // namespace

struct cs_server {
  int device = 0;
  int nslots = 0;
  int max_batch = 16;  // same-key requests a slot proves in one pass (cs_prove_batch_device)
  size_t reserve = 0;
  std::vector<cs_pk*> keys;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::thread> workers;
  bool stop = false;
  uint64_t next_id = 1;
  int busy = 0;
  size_t promised = 0;  // scratch growth admitted but not yet allocated
  // statistics
  uint64_t completed = 0, failed = 0, rejected = 0, cancelled = 0, batched = 0, batches = 0;
  uint32_t max_batch_seen = 0;
  std::vector<double> lat_ring;  // latencies (ms) of the last kLatRing completed proofs
  size_t lat_next = 0;
  int max_concurrent = 0;
  double busy_since = 0, first_start = -1, last_end = 0;
  std::string err;

  void worker(int slot);
  // Proves rq and the same-key requests in batch in one cs_prove_batch_device pass.
  int prove_group(cs_ctx* ctx, cs_pk* pk, const std::shared_ptr<Request>& rq,
                  const std::vector<std::shared_ptr<Request>>& batch, csb::PinnedBuffer& stage,
                  csb::DeviceBuffer& din, std::string& msg);
};

namespace {

// What a slot holds to prove with a set of keys: its context's scratch arena and witness
// buffer, the pinned staging of host witnesses, and the device witnesses and proofs of a
// same-key batch.
struct SlotSizes {
  size_t work = 0, in = 0, stage = 0, batch_in = 0;
};

// Batch size a slot may form for key pk (largest power of two <= max_batch, at least
// kMinBatch; 1 when the key is not batched).
uint32_t batch_cap(const cs_pk* pk, int max_batch) {
  if (max_batch < (int)kMinBatch || csb::pk_domain(pk) > (1u << 16) || !csb::pk_has_fixed(pk)) return 1;
  uint32_t k = 1;
  while (k * 2 <= (uint32_t)max_batch) k *= 2;
  return k;
}

void add_key_sizes(SlotSizes& z, const cs_pk* pk, int max_batch) {
  const size_t wbytes = (size_t)csb::pk_n_vars(pk) * 32;
  const uint32_t k = batch_cap(pk, max_batch);
  z.work = std::max(z.work, csb::prove_workspace_bytes(pk));
  z.in = std::max(z.in, wbytes + 512);
  z.stage = std::max(z.stage, wbytes * k);
  if (k > 1) z.batch_in = std::max(z.batch_in, (size_t)k * (((wbytes + 255) & ~size_t(255)) + 256));
}

SlotSizes slot_sizes(const std::vector<cs_pk*>& keys, int max_batch) {
  SlotSizes z;
  for (const cs_pk* pk : keys) add_key_sizes(z, pk, max_batch);
  return z;
}

// Device bytes a slot must still allocate to hold `want` (its buffers only grow; each adds
// an eighth of headroom when it grows).
size_t growth(const cs_ctx* ctx, const csb::DeviceBuffer& batch_in, const SlotSizes& want) {
  size_t g = 0;
  if (want.work > ctx->work.bytes) g += want.work + want.work / 8;
  if (want.in > ctx->in.bytes) g += want.in + want.in / 8;
  if (want.batch_in > batch_in.bytes) g += want.batch_in + want.batch_in / 8;
  return g;
}

}  // namespace

void cs_server::worker(int slot) {
  (void)slot;
  cudaSetDevice(device);
  cs_ctx* ctx = nullptr;
  if (cs_ctx_create(device, &ctx) != CS_OK) {
    std::lock_guard<std::mutex> lk(mu);
    err = "server slot: context creation failed";
    return;
  }
  csb::PinnedBuffer stage;
  csb::DeviceBuffer batch_in;  // witnesses and proofs of a batch
  for (;;) {
    std::shared_ptr<Request> rq;
    std::vector<std::shared_ptr<Request>> batch;  // requests proved together with rq
    size_t need = 0, batch_need = 0;
    SlotSizes grow_to;  // what the slot grows to once admitted
    {
      std::unique_lock<std::mutex> lk(mu);
      for (;;) {
        if (stop) {
          lk.unlock();
          stage.release();
          batch_in.release();
          cs_ctx_destroy(ctx);
          return;
        }
        if (!queue.empty()) {
          // A slot sizes itself for every registered key at once where memory allows, so it
          // does not grow again in steady state (growing frees the old block: a device-wide
          // synchronisation that stalls every slot); else for the head request's key alone.
          grow_to = slot_sizes(keys, max_batch);
          need = growth(ctx, batch_in, grow_to);
          if (need == 0) break;  // the slot already holds it all: nothing to admit
          size_t free_b = 0, total_b = 0;
          cudaMemGetInfo(&free_b, &total_b);
          const size_t avail = free_b > promised ? free_b - promised : 0;
          if (avail >= need + reserve) break;
          grow_to = SlotSizes{};
          add_key_sizes(grow_to, queue.front()->pk, max_batch);
          need = growth(ctx, batch_in, grow_to);
          if (need == 0 || avail >= need + reserve) break;
          if (busy == 0) {  // nothing will free memory: refuse the head request
            auto bad = queue.front();
            queue.pop_front();
            bad->status = CS_ERR_NOMEM;
            bad->err = "admission: proof scratch (" + std::to_string(need) + " bytes) does not fit in free device memory";
            bad->done = true;
            rejected++;
            cv_done.notify_all();
            continue;
          }
        }
        cv_work.wait(lk);
      }
      rq = queue.front();
      queue.pop_front();
      promised += need;
      busy++;
      if (busy > max_concurrent) max_concurrent = busy;
      rq->t_start = now_ms();
      if (first_start < 0) first_start = rq->t_start;
      // Same-key requests waiting behind it join it in one batched pass: small circuits only
      // (up to 2^16 constraints; larger proofs already fill the GPU and would only wait longer),
      // 4, 8 or 16 of them (powers of two from 4: a slot keeps few batch plans, and two or three
      // requests run as well on the other slots); plans not made yet must fit in free memory
      // (k single-proof scratches bound one).
      if (max_batch > 1 && csb::pk_domain(rq->pk) <= (1u << 16) && csb::pk_has_fixed(rq->pk)) {
        uint32_t avail_k = 1;
        for (auto& q : queue)
          if (q->pk == rq->pk && avail_k < (uint32_t)max_batch) avail_k++;
        uint32_t k = 1;
        while (k * 2 <= avail_k) k *= 2;
        if (k < kMinBatch) k = 1;
        if (k > 1 && !csb::prove_batch_ready(ctx, rq->pk, k)) {
          const size_t est = (size_t)k * (csb::prove_workspace_bytes(rq->pk) + (size_t)csb::pk_n_vars(rq->pk) * 32 + 512);
          size_t free_b = 0, total_b = 0;
          cudaMemGetInfo(&free_b, &total_b);
          const size_t fr = free_b > promised ? free_b - promised : 0;
          if (fr < est + reserve) {
            k = 1;
          } else {
            batch_need = est;  // promised until the plan exists
            promised += est;
          }
        }
        for (auto it = queue.begin(); it != queue.end() && batch.size() + 1 < k;) {
          if ((*it)->pk == rq->pk) {
            (*it)->t_start = rq->t_start;
            batch.push_back(*it);
            it = queue.erase(it);
          } else {
            ++it;
          }
        }
      }
    }
    cs_pk* pk = rq->pk;
    const size_t wbytes = (size_t)csb::pk_n_vars(pk) * 32;
    int st = CS_OK;
    std::string msg;
    if (need) {  // grow the slot's buffers now; from here on free memory accounts for them
      cudaError_t ge = csb::ctx_reserve(ctx, grow_to.work, grow_to.in);
      if (ge == cudaSuccess)
        ge = batch_in.reserve(grow_to.batch_in, static_cast<cudaStream_t>(cs_ctx_stream(ctx)));
      if (ge == cudaSuccess) ge = stage.reserve(grow_to.stage);
      {
        std::lock_guard<std::mutex> lk(mu);
        promised = promised > need ? promised - need : 0;
        need = 0;
      }
      cv_work.notify_all();
      if (ge != cudaSuccess) {
        cudaGetLastError();
        st = CS_ERR_NOMEM;
        msg = "server: slot scratch allocation failed";
      }
    }
    const size_t k = 1 + batch.size();
    if (st == CS_OK && stage.reserve(wbytes * k) != cudaSuccess) {
      st = CS_ERR_NOMEM;
      msg = "server: pinned staging buffer";
    }
    if (st == CS_OK && k == 1) {
      std::memcpy(stage.ptr, rq->w, wbytes);
      st = cs_prove(ctx, pk, static_cast<const uint32_t*>(stage.ptr), rq->r, rq->s, rq->proof);
      if (st != CS_OK) msg = cs_ctx_error(ctx);
    } else if (st == CS_OK) {
      st = prove_group(ctx, pk, rq, batch, stage, batch_in, msg);
    }
    if (batch_need) {
      std::lock_guard<std::mutex> lk(mu);
      promised = promised > batch_need ? promised - batch_need : 0;
    }
    const float dev_ms = cs_ctx_last_ms(ctx);
    {
      std::lock_guard<std::mutex> lk(mu);
      busy--;
      batch.insert(batch.begin(), rq);
      if (batch.size() > 1 && st == CS_OK) {
        batched += batch.size();
        batches++;
        max_batch_seen = std::max(max_batch_seen, (uint32_t)batch.size());
      }
      const double t_end = now_ms();
      for (auto& q : batch) {
        q->status = st;
        q->err = msg;
        q->device_ms = dev_ms;
        q->t_end = t_end;
        q->done = true;
        if (st == CS_OK) {
          completed++;
          const double lat = q->t_end - q->t_submit;
          if (lat_ring.size() < kLatRing) lat_ring.push_back(lat);
          else lat_ring[lat_next] = lat;
          lat_next = (lat_next + 1) % kLatRing;
        } else {
          failed++;
        }
      }
      last_end = t_end;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

int cs_server::prove_group(cs_ctx* ctx, cs_pk* pk, const std::shared_ptr<Request>& rq,
                           const std::vector<std::shared_ptr<Request>>& batch, csb::PinnedBuffer& stage,
                           csb::DeviceBuffer& din, std::string& msg) {
  const size_t k = 1 + batch.size();
  const size_t wbytes = (size_t)csb::pk_n_vars(pk) * 32;
  const size_t wstride = (wbytes + 255) & ~size_t(255);
  cudaStream_t st = static_cast<cudaStream_t>(cs_ctx_stream(ctx));
  cudaError_t e = din.reserve(k * wstride + k * 256, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    msg = "server: batch witness buffer";
    return CS_ERR_NOMEM;
  }
  std::vector<const uint32_t*> dw(k);
  std::vector<uint32_t*> dp(k);
  std::vector<uint32_t> r(8 * k), s(8 * k);
  char* dbase = static_cast<char*>(din.ptr);
  for (size_t i = 0; i < k; i++) {
    const Request& q = i == 0 ? *rq : *batch[i - 1];
    std::memcpy(static_cast<char*>(stage.ptr) + i * wbytes, q.w, wbytes);
    std::memcpy(&r[8 * i], q.r, 32);
    std::memcpy(&s[8 * i], q.s, 32);
    dw[i] = reinterpret_cast<const uint32_t*>(dbase + i * wstride);
    dp[i] = reinterpret_cast<uint32_t*>(dbase + k * wstride + i * 256);
    e = cudaMemcpyAsync(const_cast<uint32_t*>(dw[i]), static_cast<char*>(stage.ptr) + i * wbytes, wbytes,
                        cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      msg = "server: batch witness upload";
      cudaStreamSynchronize(st);
      cudaGetLastError();
      return CS_ERR_CUDA;
    }
  }
  int rc = cs_prove_batch_device(ctx, pk, (uint32_t)k, dw.data(), r.data(), s.data(), dp.data());
  if (rc != CS_OK) {
    msg = cs_ctx_error(ctx);
    cudaStreamSynchronize(st);  // the staged witnesses may still be in flight
    cudaGetLastError();
    return rc;
  }
  for (size_t i = 0; i < k && e == cudaSuccess; i++) {
    Request& q = i == 0 ? *rq : *batch[i - 1];
    e = cudaMemcpyAsync(q.proof, dp[i], 256, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    msg = "server: batch proof download";
    return CS_ERR_CUDA;
  }
  return CS_OK;
}

extern "C" {

int cs_server_set_max_batch(cs_server* s, int k) {
  if (!s || k < 1 || k > 64) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->max_batch = k;
  return CS_OK;
}

int cs_server_create(int device, int slots, size_t reserve_bytes, cs_server** out) {
  if (!out || slots < 1 || slots > 64) return CS_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CS_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return CS_ERR_ARG;
  std::unique_ptr<cs_server> s(new cs_server());
  s->device = device;
  s->nslots = slots;
  s->reserve = reserve_bytes;
  for (int i = 0; i < slots; i++) s->workers.emplace_back(&cs_server::worker, s.get(), i);
  *out = s.release();
  return CS_OK;
}

void cs_server_destroy(cs_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto& rq : s->queue) {
      rq->status = CS_ERR_ARG;
      rq->err = "server stopped before the request ran";
      rq->done = true;
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto& t : s->workers) t.join();
  delete s;
}

int cs_server_add_key(cs_server* s, cs_pk* pk, int* key_id) {
  if (!s || !pk || !key_id) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->keys.push_back(pk);
  *key_id = (int)s->keys.size() - 1;
  return CS_OK;
}

int cs_server_submit(cs_server* s, int key_id, const uint32_t* w, const uint32_t* r, const uint32_t* sv,
                     uint32_t* proof, uint64_t* ticket) {
  if (!s || !w || !r || !sv || !proof || !ticket) return CS_ERR_ARG;
  auto rq = std::make_shared<Request>();
  rq->key = key_id;
  rq->w = w;
  std::memcpy(rq->r, r, 32);
  std::memcpy(rq->s, sv, 32);
  rq->proof = proof;
  rq->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (key_id < 0 || key_id >= (int)s->keys.size()) return CS_ERR_ARG;
    rq->pk = s->keys[key_id];
    if (s->stop) return CS_ERR_ARG;
    rq->id = s->next_id++;
    s->live[rq->id] = rq;
    s->queue.push_back(rq);
    *ticket = rq->id;
  }
  s->cv_work.notify_one();
  return CS_OK;
}

int cs_server_wait(cs_server* s, uint64_t ticket, double timeout_s, cs_server_result* res) {
  if (!s) return CS_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(ticket);
  if (it == s->live.end()) return CS_ERR_ARG;
  auto rq = it->second;
  const auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::microseconds((long long)(timeout_s * 1e6));
  while (!rq->done) {
    if (timeout_s < 0) {
      s->cv_done.wait(lk);
    } else if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !rq->done) {
      return CS_ERR_TIMEOUT;
    }
  }
  s->live.erase(ticket);
  if (res) {
    res->status = rq->status;
    res->queue_ms = rq->t_start > 0 ? rq->t_start - rq->t_submit : 0;
    res->latency_ms = rq->t_end > 0 ? rq->t_end - rq->t_submit : 0;
    res->device_ms = rq->device_ms;
  }
  if (rq->status != CS_OK) s->err = rq->err;
  return rq->status;
}

int cs_server_stats(cs_server* s, cs_server_counters* st) {
  if (!s || !st) return CS_ERR_ARG;
  std::vector<double> lat;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    st->completed = s->completed;
    st->failed = s->failed;
    st->rejected = s->rejected;
    st->cancelled = s->cancelled;
    st->queued = s->queue.size();
    st->running = (uint32_t)s->busy;
    st->max_concurrent = (uint32_t)s->max_concurrent;
    st->promised_bytes = s->promised;
    st->batched = s->batched;
    st->batches = s->batches;
    st->max_batch_seen = s->max_batch_seen;
    lat = s->lat_ring;
  }
  st->p50_ms = st->p99_ms = 0.0;
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    st->p50_ms = lat[(size_t)(0.50 * (lat.size() - 1) + 0.5)];
    st->p99_ms = lat[(size_t)(0.99 * (lat.size() - 1) + 0.5)];
  }
  size_t free_b = 0, total_b = 0;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) cudaGetLastError();
  cudaSetDevice(prev);
  st->hbm_free_bytes = free_b;
  st->hbm_total_bytes = total_b;
  return CS_OK;
}

int cs_server_cancel(cs_server* s, uint64_t ticket) {
  if (!s) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
    if ((*it)->id == ticket) {
      (*it)->status = CS_ERR_CANCELLED;
      (*it)->err = "cancelled before it ran";
      (*it)->done = true;
      s->queue.erase(it);
      s->cancelled++;
      s->cv_done.notify_all();
      return CS_OK;
    }
  }
  return CS_ERR_ARG;  // unknown, running or finished: not cancellable
}

const char* cs_server_error(cs_server* s) { return s ? s->err.c_str() : "null server"; }

}  // extern "C"
