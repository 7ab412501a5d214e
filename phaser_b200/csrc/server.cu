// Continuous-batching request server (C ABI phgpu_server_*).
//
// Requests of any (bandwidth, voxel grid) shape are queued on submit; worker
// threads take them as soon as they are free.  Each worker owns device-resident
// contexts (tables, plans, buffers) per shape, created on demand and admitted
// against the HBM budget; an idle context of another shape is evicted when the
// budget would be exceeded.  Every worker drives its own CUDA streams, so the
// kernels of requests that arrive while others run overlap on the device.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/phaser_gpu.h"
#include "ctx.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  phgpu_params prm;
  // device-resident inputs (and host inputs under PHGPU_SERVER_BORROW_HOST)
  // are used in place: the caller keeps them alive until the ticket
  // completes; other host inputs are copied at submit
  phgpu_cloud tdev{}, sdev{};
  bool in_place = false;
  std::vector<float> txyzi, trefl, tamb, sxyzi, srefl, samb;
  uint32_t tn = 0, sn = 0;
  bool t_refl = false, t_amb = false, s_refl = false, s_amb = false;
  phgpu_pose pose;
  int status = PHGPU_OK;
  std::string err;
  Clock::time_point t_submit, t_done;
  bool done = false;
};

using ShapeKey = std::tuple<uint32_t, uint32_t, uint32_t, int32_t, int32_t, uint32_t, uint32_t, uint32_t,
                            float, float, uint32_t, uint32_t, uint32_t>;

ShapeKey key_of(const phgpu_params& p) {
  return ShapeKey(p.spherical_bandwidth, p.spherical_zero_padding, p.spatial_n_voxels,
                  p.spatial_discretize_lower, p.spatial_discretize_upper, p.n_channels, p.fusion_levels,
                  p.spherical_fusion * 2 + p.spatial_fusion, p.spatial_low_pass_lower,
                  p.spatial_low_pass_upper, p.flags, p.rot_peak_neighbors, p.trans_peak_neighbors);
}

// Device bytes of one context (upper estimate used for admission).
uint64_t estimate_bytes(const phgpu_params& p, uint32_t max_points) {
  const uint64_t bw = p.spherical_bandwidth, bo = bw + p.spherical_zero_padding, N = p.spatial_n_voxels;
  const uint64_t nv = N * N * N, H = N * N * ((N / 2 + 1 + 7) / 8 * 8);
  uint64_t b = 0;
  b += 4 * 4 * bw * bw * 2;                 // samples
  b += 8 * bw * bw * 8;                     // coef
  b += 8 * bw * 2 * bw * 8;                 // SHT scratch
  b += 8 * bo * bo * bo;                    // S
  b += 2 * 5 * nv * 4;                      // grids
  b += 9 * H * 8;                           // spec + cspec
  b += bw * bw * (bw + 1) * 4;              // Legendre table
  if ((p.flags & PHGPU_FLAG_KEEP_VOLUMES) || p.rot_peak_neighbors) b += 8 * bo * bo * bo * 4;
  if ((p.flags & PHGPU_FLAG_KEEP_VOLUMES) || p.trans_peak_neighbors) b += nv * 4;
  b += 2ull * max_points * (16 + 4 + 4 + 4 + 16 + 8 + 4 + 16) + 2ull * 32768 * 48;
  return b + (8ull << 20);
}

}  // namespace

struct phgpu_server {
  phgpu_server_params prm;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_budget;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, Request*> reqs;
  std::vector<std::thread> workers;
  uint64_t next_ticket = 1;
  uint64_t used_bytes = 0;
  size_t in_flight = 0;
  bool stop = false;
  std::string err;

  struct Owned {
    ShapeKey key;
    phgpu_ctx* ctx;
    uint64_t bytes;
  };

  void worker_main(int wid) {
    cudaSetDevice(prm.device);
    std::list<Owned> owned;  // most recently used first
    for (;;) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        if (stop && queue.empty()) break;
        r = queue.front();
        queue.pop_front();
      }
      const ShapeKey k = key_of(r->prm);
      phgpu_ctx* ctx = nullptr;
      for (auto it = owned.begin(); it != owned.end(); ++it) {
        if (it->key == k) {
          ctx = it->ctx;
          owned.splice(owned.begin(), owned, it);
          break;
        }
      }
      if (!ctx) {
        phgpu_params p = r->prm;
        p.max_points = std::max<uint32_t>(prm.max_points, std::max(r->tn, r->sn));
        p.device = prm.device;
        const uint64_t need = estimate_bytes(p, p.max_points);
        {
          std::unique_lock<std::mutex> lk(mu);
          // evict this worker's least recently used contexts until the request fits
          while (used_bytes + need > prm.hbm_budget_bytes && !owned.empty()) {
            Owned o = owned.back();
            owned.pop_back();
            lk.unlock();
            phgpu_ctx_destroy(o.ctx);
            lk.lock();
            used_bytes -= o.bytes;
            cv_budget.notify_all();
          }
          // wait for other workers to release memory
          cv_budget.wait(lk, [&] { return stop || used_bytes + need <= prm.hbm_budget_bytes || used_bytes == 0; });
          used_bytes += need;
        }
        int rc = phgpu_ctx_create(&p, &ctx);
        if (rc != PHGPU_OK) {
          std::lock_guard<std::mutex> lk(mu);
          used_bytes -= need;
          r->status = rc;
          r->err = phgpu_last_error(nullptr);
          finish(r);
          continue;
        }
        owned.push_front(Owned{k, ctx, need});
      }
      phgpu_cloud t{r->txyzi.data(), r->t_refl ? r->trefl.data() : nullptr,
                    r->t_amb ? r->tamb.data() : nullptr, r->tn, 0};
      phgpu_cloud s{r->sxyzi.data(), r->s_refl ? r->srefl.data() : nullptr,
                    r->s_amb ? r->samb.data() : nullptr, r->sn, 0};
      if (r->in_place) {
        t = r->tdev;
        s = r->sdev;
      }
      const int rc = phgpu_register_pair(ctx, &t, &s, &r->pose);
      std::lock_guard<std::mutex> lk(mu);
      r->status = rc;
      if (rc != PHGPU_OK) r->err = phgpu_last_error(ctx);
      finish(r);
    }
    std::lock_guard<std::mutex> lk(mu);
    for (auto& o : owned) {
      phgpu_ctx_destroy(o.ctx);
      used_bytes -= o.bytes;
    }
  }

  // mu held
  void finish(Request* r) {
    r->t_done = Clock::now();
    r->done = true;
    r->txyzi.clear();
    r->txyzi.shrink_to_fit();
    r->sxyzi.clear();
    r->sxyzi.shrink_to_fit();
    --in_flight;
    cv_done.notify_all();
  }
};

int phgpu_server_create(const phgpu_server_params* params, phgpu_server** out) {
  if (!params || !out) return PHGPU_ERR_INVALID;
  phgpu_server* s = new phgpu_server();
  s->prm = *params;
  if (s->prm.max_wave == 0) s->prm.max_wave = 4;
  if (s->prm.max_points == 0) s->prm.max_points = 1u << 18;
  if (s->prm.hbm_budget_bytes == 0) s->prm.hbm_budget_bytes = 150ull << 30;
  for (uint32_t w = 0; w < s->prm.max_wave; ++w) s->workers.emplace_back(&phgpu_server::worker_main, s, (int)w);
  *out = s;
  return PHGPU_OK;
}

int phgpu_server_destroy(phgpu_server* s) {
  if (!s) return PHGPU_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_budget.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
  return PHGPU_OK;
}

static void copy_cloud(const phgpu_cloud* c, std::vector<float>& xyzi, std::vector<float>& refl,
                       std::vector<float>& amb, bool& has_refl, bool& has_amb) {
  const size_t n = c->n_points;
  xyzi.resize(4 * n);
  const cudaMemcpyKind k = c->on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
  if (n) cudaMemcpy(xyzi.data(), c->xyzi, sizeof(float) * 4 * n, k);
  has_refl = c->reflectivity != nullptr;
  has_amb = c->ambient != nullptr;
  if (has_refl) {
    refl.resize(n);
    if (n) cudaMemcpy(refl.data(), c->reflectivity, sizeof(float) * n, k);
  }
  if (has_amb) {
    amb.resize(n);
    if (n) cudaMemcpy(amb.data(), c->ambient, sizeof(float) * n, k);
  }
}

int phgpu_server_submit(phgpu_server* s, const phgpu_params* params, const phgpu_cloud* target,
                        const phgpu_cloud* source, uint64_t* ticket) {
  if (!s || !params || !target || !source || !ticket) return PHGPU_ERR_INVALID;
  if (params->spatial_zero_padding != 0) {
    // the padded correlation carries state from one call to the next (the
    // previous call's last channel spectrum), so its result would depend on
    // which requests a worker context served before
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "spatial zero padding is not served (its result depends on the context's previous calls)";
    return PHGPU_ERR_INVALID;
  }
  Request* r = new Request();
  r->prm = *params;
  r->tn = target->n_points;
  r->sn = source->n_points;
  if ((target->on_device && source->on_device) || (s->prm.flags & PHGPU_SERVER_BORROW_HOST)) {
    r->in_place = true;
    r->tdev = *target;
    r->sdev = *source;
  } else {
    copy_cloud(target, r->txyzi, r->trefl, r->tamb, r->t_refl, r->t_amb);
    copy_cloud(source, r->sxyzi, r->srefl, r->samb, r->s_refl, r->s_amb);
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      return PHGPU_ERR_STATE;
    }
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->queue.push_back(r);
    ++s->in_flight;
    *ticket = r->ticket;
  }
  s->cv_work.notify_one();
  return PHGPU_OK;
}

int phgpu_server_poll(phgpu_server* s, uint64_t ticket, phgpu_pose* out, double* latency_ms) {
  if (!s) return PHGPU_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) {
    s->err = "unknown ticket";
    return PHGPU_ERR_INVALID;
  }
  Request* r = it->second;
  if (!r->done) return 0;
  if (r->status != PHGPU_OK) {
    s->err = r->err;
    const int st = r->status;
    s->reqs.erase(it);
    delete r;
    return st;
  }
  if (out) *out = r->pose;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  s->reqs.erase(it);
  delete r;
  return 1;
}

int phgpu_server_drain(phgpu_server* s) {
  if (!s) return PHGPU_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->in_flight == 0; });
  return PHGPU_OK;
}

const char* phgpu_server_last_error(const phgpu_server* s) { return s ? s->err.c_str() : ""; }
