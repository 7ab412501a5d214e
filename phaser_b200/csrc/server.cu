// Continuous-batching request server (C ABI phgpu_server_*).
//
// Requests are queued on submit.  Worker threads ("lanes") take the oldest
// request and every queued request of the same shape and channel layout, up to
// max_wave, and run them as one wave on an executor of that shape:
//
//   * an executor owns one device-resident context per slot (grids, spectra,
//     plans; point counts read from device memory) and, for the tensor-core
//     precisions, shares the shape's Wigner-d table with the other executors of
//     that bandwidth;
//   * a wave of k requests is one CUDA graph launch; an executor's first wave
//     captures the graphs of every k up to max_wave: the k pairs' front halves (target translation
//     side, sampling, SHT, fusion) on their own streams, one batched launch of
//     each SO(3) stage (synthesis on the tensor cores, angle transforms,
//     argmax) and of the pose kernel, then the k source translations, each
//     ending in one read-back of its keys and transform;
//   * the clouds are copied into the slots before the launch (device-resident
//     clouds device to device, host clouds from pinned or pageable memory).
//
// Lanes run waves concurrently, so requests that arrive while a wave is on the
// GPU are admitted into the next wave on another executor and overlap with it.
// While some wave runs, a lane holds back a wave smaller than max_wave until
// it fills or its oldest request has waited max_delay_us; an idle GPU starts a
// wave at once.
// Executors are admitted against the HBM budget with their allocators' byte
// counts; when a new one does not fit, idle executors of any shape are evicted
// (least recently used first), and a lane waits only while some other lane's
// wave holds the memory it needs -- which always finishes.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/phaser_gpu.h"
#include "ctx.h"

using namespace phgpu;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  phgpu_params prm;
  phgpu_cloud t{}, s{};  // what the worker reads (in place, or the copies below)
  std::vector<float> txyzi, trefl, tamb, sxyzi, srefl, samb;
  phgpu_pose pose;
  int status = PHGPU_OK;
  std::string err;
  Clock::time_point t_submit, t_done;
  bool done = false;
  bool want_volumes = false;
  std::vector<float> rot_vol, trans_vol;
};

using ShapeKey = std::tuple<uint32_t, uint32_t, uint32_t, int32_t, int32_t, uint32_t, uint32_t, uint32_t, float,
                            float, uint32_t, uint32_t, uint32_t, uint32_t, uint32_t, uint32_t, int>;

// Everything that decides a wave's buffers and captured graph: the shape and
// fusion parameters and which optional channels each cloud carries.
ShapeKey key_of(const phgpu_params& p, const phgpu_cloud& t, const phgpu_cloud& s) {
  const int sig = (t.reflectivity ? 1 : 0) | (t.ambient ? 2 : 0) | (s.reflectivity ? 4 : 0) | (s.ambient ? 8 : 0);
  return ShapeKey(p.spherical_bandwidth, p.spherical_zero_padding, p.spatial_n_voxels, p.spatial_discretize_lower,
                  p.spatial_discretize_upper, p.n_channels, p.fusion_levels, p.spherical_fusion * 4 + p.spatial_fusion,
                  p.spatial_low_pass_lower, p.spatial_low_pass_upper, p.flags & PHGPU_FLAG_KEEP_VOLUMES,
                  p.rot_peak_neighbors, p.trans_peak_neighbors,
                  p.spherical_low_pass_lower, p.spherical_low_pass_upper, p.precision, sig);
}

// Device bytes of one slot before any exists (an upper estimate; executors
// are then accounted with their allocators' counts).
uint64_t estimate_slot_bytes(const phgpu_params& p, uint32_t max_points) {
  const uint64_t bw = p.spherical_bandwidth, bo = bw + p.spherical_zero_padding, N = p.spatial_n_voxels;
  const uint64_t nv = N * N * N, H = N * N * ((N / 2 + 1 + 7) / 8 * 8);
  uint64_t b = 0;
  b += 4 * 4 * bw * bw * 2 + 8 * bw * bw * 8 + 8 * bw * 2 * bw * 8;  // samples, coefficients, SHT scratch
  b += 8 * bo * bo * bo;                                           // S
  b += 2 * 5 * nv * 4 + 9 * H * 8;                                 // grids, spectra
  b += bw * bw * (bw + 1) * 4;                                     // Legendre table
  if (p.flags & PHGPU_FLAG_KEEP_VOLUMES || p.rot_peak_neighbors) b += 8 * bo * bo * bo * 4;
  if (p.flags & PHGPU_FLAG_KEEP_VOLUMES || p.trans_peak_neighbors) b += nv * 4;
  b += 2ull * max_points * (16 + 4 + 4 + 4 + 16 + 8 + 4 + 16) + 2ull * 32768 * 48;
  return b + (8ull << 20);
}

// A Wigner-d table shared by the executors of one (bandwidth, output bandwidth).
struct Table {
  float* d_tab = nullptr;
  size_t* d_off = nullptr;
  uint64_t bytes = 0;
  int refs = 0;
};

struct Executor {
  ShapeKey key;
  phgpu_params prm;
  PairPlan pp{};
  int kmax = 1;
  bool graphs = true;  // waves replay captured graphs (device pose path)
  std::vector<phgpu_ctx*> slots;
  cudaStream_t st = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_mid = nullptr, ev_done = nullptr;
  std::vector<cudaEvent_t> ev_join;
  std::vector<cudaGraphExec_t> exec;  // [k] wave of k requests
  std::vector<int> capture_failures;  // [k] captures of a k-request wave that were invalidated
  std::vector<unsigned long long> graph_kernels;  // [k] kernels in the graph of a k-request wave
  std::shared_ptr<Table> table;
  uint64_t bytes = 0;
  bool busy = false;
  bool captured_all = false;  // the graphs of every wave size were captured (first wave)
  Clock::time_point last_used;
};

}  // namespace

struct phgpu_server {
  phgpu_server_params prm;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_budget;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, Request*> reqs;
  std::vector<std::thread> workers;
  std::vector<std::unique_ptr<Executor>> execs;
  std::map<std::pair<uint32_t, uint32_t>, std::weak_ptr<Table>> tables;
  std::map<ShapeKey, uint64_t> measured_bytes;  // bytes of an executor of each key (allocator counts)
  // Held while a lane captures a wave graph and while an executor is created or
  // destroyed: allocation, frees and synchronous set-up calls synchronise the
  // device, which would invalidate a capture running in another lane.
  std::mutex cuda_excl;
  // tunings by (bandwidth, spherical zero padding, voxels, precision)
  std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, phgpu_tuning> tunings;
  uint64_t next_ticket = 1;
  uint64_t used_bytes = 0;
  size_t in_flight = 0;
  int running = 0;  // lanes running a wave
  bool stop = false;
  std::string err;
  phgpu_server_stats stats{};

  // ---------------------------------------------------------------- executors

  // mu held on entry and exit; released while CUDA objects are created.
  Executor* acquire(const ShapeKey& key, const phgpu_params& rp, int want, std::unique_lock<std::mutex>& lk,
                    int* rc, std::string* why) {
    for (;;) {
      for (auto& e : execs)
        if (!e->busy && e->key == key) {
          e->busy = true;
          return e.get();
        }
      const int kmax = std::max(1, std::min<int>((int)prm.max_wave, kMaxWave));
      auto mb = measured_bytes.find(key);
      const uint64_t need =
          mb != measured_bytes.end() ? mb->second : estimate_slot_bytes(rp, prm.max_points) * (uint64_t)kmax;
      // evict idle executors (any shape, least recently used first) until the new one fits
      while (used_bytes + need > prm.hbm_budget_bytes) {
        Executor* lru = nullptr;
        for (auto& e : execs)
          if (!e->busy && (!lru || e->last_used < lru->last_used)) lru = e.get();
        if (!lru) break;
        lru->busy = true;
        lk.unlock();
        {
          std::lock_guard<std::mutex> ex(cuda_excl);
          destroy_exec(lru);
        }
        lk.lock();
        used_bytes -= lru->bytes;
        execs.erase(std::find_if(execs.begin(), execs.end(), [&](auto& e) { return e.get() == lru; }));
        ++stats.evictions;
      }
      if (used_bytes + need <= prm.hbm_budget_bytes || used_bytes == 0) {
        used_bytes += need;  // reserved; corrected to the allocators' count below
        auto ex = std::make_unique<Executor>();
        Executor* e = ex.get();
        e->key = key;
        e->prm = rp;
        e->busy = true;
        e->kmax = kmax;
        execs.push_back(std::move(ex));
        lk.unlock();
        int r;
        {
          std::lock_guard<std::mutex> ex(cuda_excl);
          r = create_exec(e, why);
        }
        lk.lock();
        used_bytes -= need;
        if (r != PHGPU_OK) {
          execs.erase(std::find_if(execs.begin(), execs.end(), [&](auto& x) { return x.get() == e; }));
          *rc = r;
          cv_budget.notify_all();
          return nullptr;
        }
        used_bytes += e->bytes;
        measured_bytes[key] = e->bytes;
        return e;
      }
      // every executor is busy in another lane's wave: wait for one to finish
      cv_budget.wait(lk);
      if (stop) {
        *rc = PHGPU_ERR_STATE;
        *why = "server stopped";
        return nullptr;
      }
    }
    (void)want;
  }

  void release(Executor* e) {
    e->busy = false;
    e->last_used = Clock::now();
    cv_budget.notify_all();
  }

  int create_exec(Executor* e, std::string* why) {
    cudaSetDevice(prm.device);
    phgpu_params p = e->prm;
    p.max_points = prm.max_points;
    p.device = prm.device;
    // slots keep the request's precision (tensor-core Legendre tables of their
    // own); the executor holds the shape's Wigner-d table
    const int bw_out = (int)(p.spherical_bandwidth + p.spherical_zero_padding);
    if (e->prm.precision != PHGPU_PRECISION_FP32)
      while (e->kmax > 1 && (!so3_tc_supported(bw_out, e->kmax, (int)e->prm.precision) ||
                             !sht_leg_tc_supported((int)p.spherical_bandwidth, e->kmax, (int)e->prm.precision)))
        --e->kmax;
    e->graphs = e->prm.rot_peak_neighbors == 0 && e->prm.spatial_zero_padding == 0;
    for (int i = 0; i < e->kmax; ++i) {
      phgpu_ctx* c = nullptr;
      const int rc = phgpu_ctx_create_internal(&p, &c, false);
      if (rc != PHGPU_OK) {
        *why = phgpu_last_error(nullptr);
        destroy_exec(e);
        return rc;
      }
      e->slots.push_back(c);
      e->bytes += c->device_bytes;
      {
        std::lock_guard<std::mutex> lk(mu);
        auto it = tunings.find(std::make_tuple(p.spherical_bandwidth, p.spherical_zero_padding, p.spatial_n_voxels,
                                               e->prm.precision));
        if (it != tunings.end()) phgpu_tuning_set(c, &it->second);
      }
      // point counts from device memory (any count up to the capacity replays
      // the same graph); grids zeroed once, the graph's clears keep them so
      c->dev_counts = true;
      const size_t nv = (size_t)c->N * c->N * c->N;
      for (int s = 0; s < 2; ++s) {
        if (cudaMemset(c->d_grids[s], 0, sizeof(float) * 5 * nv) != cudaSuccess ||
            cudaMemset(c->d_rowlive[s], 0, (size_t)c->N * c->N) != cudaSuccess) {
          *why = "grid initialisation failed";
          destroy_exec(e);
          return PHGPU_ERR_CUDA;
        }
        c->clean_planes[s] = 5;
      }
    }
    if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_mid, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_done, cudaEventDisableTiming) != cudaSuccess) {
      *why = "stream / event creation failed";
      destroy_exec(e);
      return PHGPU_ERR_CUDA;
    }
    e->ev_join.assign(e->kmax, nullptr);
    for (auto& ev : e->ev_join) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    e->exec.assign(e->kmax + 1, nullptr);
    if (e->prm.precision != PHGPU_PRECISION_FP32) {
      const int rc = attach_table(e, why);
      if (rc != PHGPU_OK) {
        destroy_exec(e);
        return rc;
      }
    }
    if (cudaStreamSynchronize(e->st) != cudaSuccess) {
      *why = "executor set-up failed";
      destroy_exec(e);
      return PHGPU_ERR_CUDA;
    }
    e->capture_failures.assign(e->kmax + 1, 0);
    e->graph_kernels.assign(e->kmax + 1, 0);
    return PHGPU_OK;
  }

  // The shape's Wigner-d table, shared with other executors of the bandwidth.
  int attach_table(Executor* e, std::string* why) {
    phgpu_ctx* c = e->slots[0];
    const auto tk = std::make_pair((uint32_t)c->bw, (uint32_t)c->bw_out);
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = tables.find(tk);
      if (it != tables.end()) e->table = it->second.lock();
    }
    if (e->table) return PHGPU_OK;
    auto t = std::make_shared<Table>();
    std::vector<size_t> off;
    const size_t nf = so3_table_layout(c->bw, c->bw_out, &off);
    if (cudaMalloc((void**)&t->d_off, sizeof(size_t) * off.size()) != cudaSuccess ||
        cudaMalloc((void**)&t->d_tab, sizeof(float) * nf) != cudaSuccess) {
      if (t->d_off) cudaFree(t->d_off);
      *why = "Wigner-d table allocation failed";
      return PHGPU_ERR_MEMORY;
    }
    t->bytes = sizeof(size_t) * off.size() + sizeof(float) * nf;
    if (cudaMemcpy(t->d_off, off.data(), sizeof(size_t) * off.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        launch_so3_table(c->bw, c->bw_out, c->d_beta_tab, c->d_wig_tab, t->d_off, t->d_tab, e->st) != cudaSuccess) {
      cudaFree(t->d_off);
      cudaFree(t->d_tab);
      *why = "Wigner-d table generation failed";
      return PHGPU_ERR_CUDA;
    }
    e->bytes += t->bytes;
    e->table = t;
    std::lock_guard<std::mutex> lk(mu);
    tables[tk] = t;
    return PHGPU_OK;
  }

  void destroy_exec(Executor* e) {
    cudaSetDevice(prm.device);
    if (e->st) cudaStreamSynchronize(e->st);
    for (auto& g : e->exec)
      if (g) cudaGraphExecDestroy(g);
    e->exec.clear();
    for (auto* c : e->slots) phgpu_ctx_destroy(c);
    e->slots.clear();
    for (auto& ev : e->ev_join)
      if (ev) cudaEventDestroy(ev);
    e->ev_join.clear();
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_mid) cudaEventDestroy(e->ev_mid);
    if (e->ev_done) cudaEventDestroy(e->ev_done);
    if (e->st) cudaStreamDestroy(e->st);
    e->ev_fork = e->ev_mid = e->ev_done = nullptr;
    e->st = nullptr;
    if (e->table) {
      if (e->table.use_count() == 1) {
        cudaFree(e->table->d_tab);
        cudaFree(e->table->d_off);
      }
      e->table.reset();
    }
  }

  // ---------------------------------------------------------------- waves

  // Enqueues a wave of k requests already staged in slots [0, k) on the
  // executor's streams (captured into a graph, or run directly).
  int enqueue_wave(Executor* e, int k) {
    std::vector<phgpu_ctx*> sl(e->slots.begin(), e->slots.begin() + k);
    phgpu_ctx* c0 = sl[0];
    if (cudaEventRecord(e->ev_fork, e->st) != cudaSuccess) return PHGPU_ERR_CUDA;
    // tensor-core precisions: the fronts stop after the phi transform and the
    // Legendre contraction and the fusion run once for the whole wave
    const bool batch_leg = e->table != nullptr;
    for (int i = 0; i < k; ++i) {
      if (cudaStreamWaitEvent(sl[i]->s0, e->ev_fork, 0) != cudaSuccess) return PHGPU_ERR_CUDA;
      const int rc = phgpu_pair_front(sl[i], e->pp, batch_leg);
      if (rc != PHGPU_OK) return rc;
      if (cudaEventRecord(e->ev_join[i], sl[i]->s0) != cudaSuccess ||
          cudaStreamWaitEvent(e->st, e->ev_join[i], 0) != cudaSuccess)
        return PHGPU_ERR_CUDA;
    }
    if (batch_leg) {
      const int rc = phgpu_run_sph_leg_fuse_batch(sl.data(), k, e->pp.laplace_s2 ? e->pp.nd_s2 : 1,
                                                  (int)c0->prm.n_channels, e->pp.laplace_s2,
                                                  c0->prm.spherical_fusion == PHGPU_FUSION_MIX, e->st);
      if (rc != PHGPU_OK) return rc;
    }
    So3Table tab;
    if (e->table) {
      tab.table = e->table->d_tab;
      tab.class_off = e->table->d_off;
      tab.precision = (int)e->prm.precision;
    }
    int rc = phgpu_run_so3_batch(sl.data(), k, e->table ? &tab : nullptr, e->st);
    if (rc != PHGPU_OK) return rc;
    PoseBatch pb;
    memset(&pb, 0, sizeof(pb));
    pb.count = k;
    pb.bw_out = (uint32_t)c0->bw_out;
    for (int i = 0; i < k; ++i) {
      pb.argmax[i] = sl[i]->d_argmax;
      pb.T[i] = sl[i]->d_T;
    }
    if (launch_pose(pb, e->st) != cudaSuccess || cudaEventRecord(e->ev_mid, e->st) != cudaSuccess)
      return PHGPU_ERR_CUDA;
    for (int i = 0; i < k; ++i) {
      if (cudaStreamWaitEvent(sl[i]->s0, e->ev_mid, 0) != cudaSuccess) return PHGPU_ERR_CUDA;
      rc = phgpu_pair_back(sl[i], e->pp, nullptr, sl[i]->d_T);
      if (rc != PHGPU_OK) return rc;
      if (cudaEventRecord(e->ev_join[i], sl[i]->s0) != cudaSuccess ||
          cudaStreamWaitEvent(e->st, e->ev_join[i], 0) != cudaSuccess)
        return PHGPU_ERR_CUDA;
    }
    return PHGPU_OK;
  }

  int capture(Executor* e, int k, std::string* why) {
    std::lock_guard<std::mutex> ex(cuda_excl);
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      *why = "stream capture could not start";
      return PHGPU_ERR_CUDA;
    }
    ++g_capture_depth;
    const int rc = enqueue_wave(e, k);
    --g_capture_depth;
    const cudaError_t ce = cudaStreamEndCapture(e->st, &g);
    // the graph's kernels run (and are counted) at each replay
    unsigned long long kernels = 0;
    size_t nn = 0;
    if (g && cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn) {
      std::vector<cudaGraphNode_t> nodes(nn);
      cudaGraphGetNodes(g, nodes.data(), &nn);
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++kernels;
      }
    }
    e->graph_kernels[k] = kernels;
    if (rc != PHGPU_OK || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      *why = rc != PHGPU_OK ? std::string("wave capture: ") + phgpu_last_error(e->slots[0])
                            : std::string("wave capture: ") + cudaGetErrorString(ce);
      cudaGetLastError();
      return PHGPU_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&e->exec[k], g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      e->exec[k] = nullptr;
      *why = std::string("graph instantiation: ") + cudaGetErrorString(ie);
      return PHGPU_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(mu);
    ++stats.graph_captures;
    return PHGPU_OK;
  }

  void run_wave(Executor* e, std::vector<Request*>& wave) {
    cudaSetDevice(prm.device);
    const int k = (int)wave.size();
    std::string why;
    int rc = PHGPU_OK;
    e->pp = pair_plan(e->slots[0], wave[0]->t.reflectivity, wave[0]->t.ambient, wave[0]->s.reflectivity,
                      wave[0]->s.ambient);
    if (!e->graphs) {
      // host-pose registrations (peak neighbourhoods): one at a time
      for (int i = 0; i < k; ++i) {
        Request* r = wave[i];
        r->status = phgpu_register_pair(e->slots[0], &r->t, &r->s, &r->pose);
        if (r->status != PHGPU_OK) r->err = phgpu_last_error(e->slots[0]);
        if (r->status == PHGPU_OK && r->want_volumes) copy_volumes(e->slots[0], r);
      }
      std::lock_guard<std::mutex> lk(mu);
      ++stats.waves;
      stats.requests += (uint64_t)k;
      return;
    }
    for (int i = 0; i < k && rc == PHGPU_OK; ++i) {
      rc = phgpu_upload_cloud(e->slots[i], &wave[i]->t, 0, e->st);
      if (rc == PHGPU_OK) rc = phgpu_upload_cloud(e->slots[i], &wave[i]->s, 1, e->st);
      if (rc != PHGPU_OK) why = phgpu_last_error(e->slots[i]);
    }
    // the first wave of an executor captures the graphs of every wave size, so
    // no later wave waits for a capture; CUDA work of other threads of the
    // process that synchronises the device invalidates a capture, so after a
    // failed capture the wave runs uncaptured (the same launches) and capturing
    // is retried on later waves (twice at most)
    if (rc == PHGPU_OK && !e->captured_all) {
      e->captured_all = true;
      // a captured launch keeps the optional-channel pointers its slot had at
      // capture time: slots this wave leaves empty take the channel layout
      // every request of the executor's key has
      for (int i = k; i < e->kmax; ++i)
        for (int sd = 0; sd < 2; ++sd) {
          e->slots[i]->has_refl[sd] = e->slots[0]->has_refl[sd];
          e->slots[i]->has_amb[sd] = e->slots[0]->has_amb[sd];
        }
      for (int kk = 1; kk <= e->kmax; ++kk) {
        std::string ignore;
        if (!e->exec[kk] && capture(e, kk, &ignore) != PHGPU_OK) {
          ++e->capture_failures[kk];
          cudaGetLastError();
        }
      }
    }
    bool direct = false;
    if (rc == PHGPU_OK && !e->exec[k]) {
      if (e->capture_failures[k] < 2 && capture(e, k, &why) == PHGPU_OK) {
        why.clear();
      } else {
        ++e->capture_failures[k];
        direct = true;
        why.clear();
        cudaGetLastError();
      }
    }
    if (rc == PHGPU_OK) {
      cudaError_t ce = cudaSuccess;
      if (direct) {
        rc = enqueue_wave(e, k);
        if (rc != PHGPU_OK) why = phgpu_last_error(e->slots[0]);
      } else {
        ce = cudaGraphLaunch(e->exec[k], e->st);
        count_launches((int)e->graph_kernels[k]);
      }
      if (rc == PHGPU_OK && ce == cudaSuccess) ce = cudaEventRecord(e->ev_done, e->st);
      if (rc == PHGPU_OK && ce == cudaSuccess) ce = cudaEventSynchronize(e->ev_done);
      if (rc == PHGPU_OK && ce != cudaSuccess) {
        rc = PHGPU_ERR_CUDA;
        why = std::string("wave: ") + cudaGetErrorString(ce);
      }
      if (direct) {
        std::lock_guard<std::mutex> lk(mu);
        ++stats.direct_waves;
      }
    }
    uint64_t reruns = 0;
    for (int i = 0; i < k; ++i) {
      Request* r = wave[i];
      if (rc != PHGPU_OK) {
        r->status = rc;
        r->err = why;
        continue;
      }
      phgpu_ctx* c = e->slots[i];
      const uint64_t before = c->pose_reruns;
      r->status = phgpu_pair_finish(c, e->pp, true, &r->pose);
      reruns += c->pose_reruns - before;
      if (r->status != PHGPU_OK) r->err = phgpu_last_error(c);
      if (r->status == PHGPU_OK && r->want_volumes) copy_volumes(c, r);
    }
    std::lock_guard<std::mutex> lk(mu);
    ++stats.waves;
    stats.requests += (uint64_t)k;
    stats.pose_reruns += reruns;
  }

  static void copy_volumes(phgpu_ctx* c, Request* r) {
    const size_t nr = (size_t)8 * c->bw_out * c->bw_out * c->bw_out;
    const size_t nt = (size_t)c->N * c->N * c->N;
    r->rot_vol.resize(nr);
    r->trans_vol.resize(nt);
    if (c->d_rotvol) cudaMemcpy(r->rot_vol.data(), c->d_rotvol, sizeof(float) * nr, cudaMemcpyDeviceToHost);
    if (c->d_transvol) cudaMemcpy(r->trans_vol.data(), c->d_transvol, sizeof(float) * nt, cudaMemcpyDeviceToHost);
  }

  void worker_main() {
    cudaSetDevice(prm.device);
    for (;;) {
      std::vector<Request*> wave;
      ShapeKey key;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        if (stop && queue.empty()) break;
        const size_t kmax = std::max<uint32_t>(1u, std::min<uint32_t>(prm.max_wave, kMaxWave));
        // Dynamic batching: while another lane's wave is on the GPU, a partial
        // wave is held back so the queue can fill it -- until the oldest
        // request's shape has max_wave requests queued, no wave runs, or the
        // oldest request has waited max_delay_us.  An idle GPU starts at once.
        for (;;) {
          if (stop || queue.empty()) break;
          const ShapeKey k0 = key_of(queue.front()->prm, queue.front()->t, queue.front()->s);
          size_t same = 0;
          for (Request* r : queue)
            if (key_of(r->prm, r->t, r->s) == k0 && ++same >= kmax) break;
          if (same >= kmax || running == 0) break;
          const auto waited = Clock::now() - queue.front()->t_submit;
          const auto limit = std::chrono::microseconds(prm.max_delay_us);
          if (waited >= limit) break;
          cv_work.wait_for(lk, limit - waited);
        }
        if (queue.empty()) {
          if (stop) break;
          continue;
        }
        // the oldest request and every queued request of its key, up to max_wave
        Request* first = queue.front();
        key = key_of(first->prm, first->t, first->s);
        for (auto it = queue.begin(); it != queue.end() && wave.size() < kmax;) {
          if (key_of((*it)->prm, (*it)->t, (*it)->s) == key) {
            wave.push_back(*it);
            it = queue.erase(it);
          } else {
            ++it;
          }
        }
        int rc = PHGPU_OK;
        std::string why;
        Executor* e = acquire(key, first->prm, (int)wave.size(), lk, &rc, &why);
        if (!e) {
          for (Request* r : wave) {
            r->status = rc;
            r->err = why;
            finish(r);
          }
          continue;
        }
        // an executor may hold fewer slots than the wave (shared / tensor memory)
        if ((int)wave.size() > e->kmax) {
          for (size_t i = wave.size(); i-- > (size_t)e->kmax;) queue.push_front(wave[i]);
          wave.resize(e->kmax);
          cv_work.notify_one();
        }
        ++running;
        lk.unlock();
        run_wave(e, wave);
        lk.lock();
        --running;
        cv_work.notify_all();
        release(e);
        for (Request* r : wave) finish(r);
      }
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
  if (s->prm.max_wave == 0) s->prm.max_wave = 16;
  if (s->prm.max_wave > (uint32_t)kMaxWave) s->prm.max_wave = kMaxWave;
  if (s->prm.max_points == 0) s->prm.max_points = 1u << 18;
  if (s->prm.hbm_budget_bytes == 0) s->prm.hbm_budget_bytes = 150ull << 30;
  if (s->prm.lanes == 0) s->prm.lanes = 2;
  if (s->prm.max_delay_us == 0) s->prm.max_delay_us = 500;
  for (uint32_t w = 0; w < s->prm.lanes; ++w) s->workers.emplace_back(&phgpu_server::worker_main, s);
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
  for (auto& e : s->execs) s->destroy_exec(e.get());
  s->execs.clear();
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
  return PHGPU_OK;
}

static void copy_cloud(const phgpu_cloud* c, std::vector<float>& xyzi, std::vector<float>& refl,
                       std::vector<float>& amb, phgpu_cloud* dst) {
  const size_t n = c->n_points;
  xyzi.resize(4 * n);
  const cudaMemcpyKind k = c->on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
  if (n) cudaMemcpy(xyzi.data(), c->xyzi, sizeof(float) * 4 * n, k);
  if (c->reflectivity) {
    refl.resize(n);
    if (n) cudaMemcpy(refl.data(), c->reflectivity, sizeof(float) * n, k);
  }
  if (c->ambient) {
    amb.resize(n);
    if (n) cudaMemcpy(amb.data(), c->ambient, sizeof(float) * n, k);
  }
  *dst = phgpu_cloud{xyzi.data(), c->reflectivity ? refl.data() : nullptr, c->ambient ? amb.data() : nullptr,
                     c->n_points, 0};
}

int phgpu_server_submit(phgpu_server* s, const phgpu_params* params, const phgpu_cloud* target,
                        const phgpu_cloud* source, uint64_t* ticket) {
  if (!s || !params || !target || !source || !ticket) return PHGPU_ERR_INVALID;
  if (params->spatial_zero_padding != 0) {
    // the padded correlation carries state from one call to the next (the
    // previous call's last channel spectrum), so its result would depend on
    // which requests a slot served before
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "spatial zero padding is not served (its result depends on the context's previous calls)";
    return PHGPU_ERR_INVALID;
  }
  if (target->n_points > s->prm.max_points || source->n_points > s->prm.max_points) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "cloud larger than the server's max_points";
    return PHGPU_ERR_LIMIT;
  }
  if (target->on_device != source->on_device) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "both clouds must be on the device or both on the host";
    return PHGPU_ERR_INVALID;
  }
  Request* r = new Request();
  r->prm = *params;
  r->want_volumes = (params->flags & PHGPU_FLAG_KEEP_VOLUMES) != 0;
  if (target->on_device || (s->prm.flags & PHGPU_SERVER_BORROW_HOST)) {
    r->t = *target;
    r->s = *source;
  } else {
    copy_cloud(target, r->txyzi, r->trefl, r->tamb, &r->t);
    copy_cloud(source, r->sxyzi, r->srefl, r->samb, &r->s);
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

int phgpu_server_poll_volumes(phgpu_server* s, uint64_t ticket, phgpu_pose* out, double* latency_ms,
                              float* rot_volume, float* trans_volume) {
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
  if ((rot_volume || trans_volume) && !r->want_volumes) {
    s->err = "volumes were not kept (submit with PHGPU_FLAG_KEEP_VOLUMES)";
    return PHGPU_ERR_STATE;
  }
  if (rot_volume) memcpy(rot_volume, r->rot_vol.data(), sizeof(float) * r->rot_vol.size());
  if (trans_volume) memcpy(trans_volume, r->trans_vol.data(), sizeof(float) * r->trans_vol.size());
  if (out) *out = r->pose;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  s->reqs.erase(it);
  delete r;
  return 1;
}

int phgpu_server_poll(phgpu_server* s, uint64_t ticket, phgpu_pose* out, double* latency_ms) {
  return phgpu_server_poll_volumes(s, ticket, out, latency_ms, nullptr, nullptr);
}

int phgpu_server_drain(phgpu_server* s) {
  if (!s) return PHGPU_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->in_flight == 0; });
  return PHGPU_OK;
}

int phgpu_server_get_stats(phgpu_server* s, phgpu_server_stats* out) {
  if (!s || !out) return PHGPU_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->executors = (uint64_t)s->execs.size();
  out->bytes_in_use = s->used_bytes;
  return PHGPU_OK;
}

int phgpu_server_set_tuning(phgpu_server* s, const phgpu_params* shape, const phgpu_tuning* t) {
  if (!s || !shape || !t) return PHGPU_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  s->tunings[std::make_tuple(shape->spherical_bandwidth, shape->spherical_zero_padding, shape->spatial_n_voxels,
                             shape->precision)] = *t;
  return PHGPU_OK;
}

const char* phgpu_server_last_error(const phgpu_server* s) { return s ? s->err.c_str() : ""; }
