// Render-serving loop (include/appearance_cuda.h, "serving"): resident scenes,
// jobs of mixed resolution / samples / scene admitted as device memory and
// execution slots free up, and run concurrently, each on its own stream.
//
// The reference serves frames through a synchronous frame farm (Host/Node,
// crates/appearance-render-loop/src/host.rs:250-505, node.rs:27-147): one
// resident renderer per node renders the rows it is asked for, one request at
// a time.  Here one process owns the GPU and keeps every scene's BVH and
// tables resident; a dispatcher thread admits queued jobs in arrival order
// while their frame state fits the device-memory budget and a slot is free,
// allocates that state from the stream-ordered pool (cudaMallocAsync, no
// device-wide synchronisation), and launches the job's frame (the same
// encode_frame as ap_render_*) on the slot's stream, optionally as a CUDA graph
// captured once per job shape and updated in place for later jobs.  Jobs in
// flight overlap on the device; a host callback on each stream wakes the
// dispatcher when a job's result has reached host memory.  With a plain
// estimator configuration, jobs waiting with the same sample and bounce
// counts are admitted together as one batch of up to kMaxBatch frames: the
// batch runs as one launch sequence (encode_batch_plain) whose traversal
// stages are single persistent launches over all its frames' ray queues.  A
// job's result is a function of its own inputs only (its seed, camera, scene
// and sizes), so it is the same alone, batched and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/appearance_cuda.h"
#include "device_scope.h"
#include "frame.cuh"

namespace ap {
int handle_trace_context(void* hp, const DevScene** scene, const TwoLevel** two_level, cudaStream_t* stream,
                         int* num_sms, int* device, std::string** err);
size_t handle_scene_bytes(void* hp);
}  // namespace ap

namespace {

using namespace ap;
using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
  uint64_t ticket = 0;
  ap_job desc{};
  float* out = nullptr;
  bool out_pinned = false;
  Clock::time_point t_submit, t_admit, t_done;
  int slot = -1;
  void* dev = nullptr;
  size_t bytes = 0;
  bool done = false;
  int rc = AP_OK;
  std::string err;
  double gpu_ms = 0.0;
  int graph_mode = 0;  // 0 direct launches, 1 graph instantiated, 2 graph updated in place
  bool cancelled = false;
  int batch = 1;  // frames of the launch sequence the job ran in
  float* staging = nullptr;  // its slot's pinned result buffer (pageable callers)
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // pinned, per batch position, for callers whose output buffer is pageable
  float* staging[kMaxBatch] = {};
  size_t staging_bytes[kMaxBatch] = {};
  JobTrace* h_table = nullptr;  // pinned: the batch's traversal table, copied to d_table in the stream
  JobTrace* d_table = nullptr;
  // instantiated frame graphs of this slot, one per launch sequence (shape
  // key); a later job of the same key updates its graph in place
  std::map<uint64_t, cudaGraphExec_t> execs;
  std::vector<Job*> jobs;  // the batch in flight; empty when the slot is free
  bool finished = false;   // set by the stream callback
};

struct Server {
  int device = 0;
  int num_sms = 148;
  uint64_t budget = 0;
  int use_graphs = 0;
  uint32_t max_batch = kMaxBatch;  // ap_server_set_batching
  FrameConfig base{};
  std::vector<void*> scenes;
  size_t scene_bytes = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> pending;
  std::map<uint64_t, Job*> jobs;
  std::vector<Slot> slots;
  size_t in_use = 0, peak = 0;
  uint64_t next_ticket = 1, completed = 0;
  std::atomic<uint64_t> graph_updates{0}, graph_instantiations{0};  // written by the dispatcher
  bool stop = false;
  std::thread worker;
  std::string err;
  cudaMemPool_t pool = nullptr;  // the server's own stream-ordered pool
};

struct CallbackArg {
  Server* srv;
  int slot;
};

void CUDART_CB on_slot_done(void* p) {  // runs on a CUDA callback thread: no CUDA calls here
  CallbackArg* a = static_cast<CallbackArg*>(p);
  {
    std::lock_guard<std::mutex> lk(a->srv->mu);
    a->srv->slots[a->slot].finished = true;
  }
  a->srv->cv_work.notify_one();
  delete a;
}

uint64_t shape_key(const FrameConfig& cfg, int batch) {
  // the launch sequence depends on the sample and bounce counts and the batch
  // size only; resolutions, scenes, cameras and buffers are node parameters,
  // which an in-place update may change
  uint64_t k = 1469598103934665603ull;
  auto mix = [&](uint64_t v) { k = (k ^ v) * 1099511628211ull; };
  mix(cfg.sample_count);
  mix(cfg.max_bounces);
  mix((uint64_t)batch);
  return k;
}

// Jobs that may share a launch sequence.
bool same_shape(const ap_job& a, const ap_job& b) { return a.spp == b.spp && a.max_depth == b.max_depth; }

// Enqueues the admitted batch on the slot's stream (dispatcher thread, no
// lock held).  The jobs enqueued go to `ok`; those whose frame state cannot be
// allocated go to `failed` (rc set).  Returns false when nothing was enqueued.
bool launch_batch(Server* s, Slot& sl, const std::vector<Job*>& batch, std::vector<Job*>* ok_out,
                  std::vector<Job*>* failed) {
  FrameConfig cfg = s->base;
  cfg.sample_count = batch[0]->desc.spp;
  cfg.max_bounces = batch[0]->desc.max_depth;
  std::vector<Job*>& ok = *ok_out;
  BatchFrame frames[kMaxBatch];
  for (Job* j : batch) {
    const ap_job& d = j->desc;
    cudaError_t e = cudaMallocFromPoolAsync(&j->dev, j->bytes, s->pool, sl.stream);
    if (e != cudaSuccess) {
      j->rc = e == cudaErrorMemoryAllocation ? AP_E_OOM : AP_E_CUDA;
      j->err = std::string("job frame state: ") + cudaGetErrorString(e);
      j->dev = nullptr;
      cudaGetLastError();
      failed->push_back(j);
      continue;
    }
    cudaMemsetAsync(j->dev, 0, j->bytes, sl.stream);  // a job starts from a fresh frame sequence
    const DevScene* scene = nullptr;
    cudaStream_t unused_stream;
    const TwoLevel* unused_two_level = nullptr;  // server scenes are flat uploads
    int sms = 0, dev = 0;
    std::string* err = nullptr;
    ap::handle_trace_context(s->scenes[d.scene], &scene, &unused_two_level, &unused_stream, &sms, &dev, &err);
    BatchFrame& f = frames[ok.size()];
    f.scene = *scene;
    frame_buffers_carve(j->dev, d.width, d.height, &f.fb);
    std::memcpy(&f.mats, d.mats, sizeof(Mats));
    f.W = d.width;
    f.H = d.height;
    f.frame_idx = d.seed;
    ok.push_back(j);
  }
  const int nj = (int)ok.size();
  if (nj == 0) return false;
  const bool batched = nj > 1;
  for (int k = 0; k < nj; ++k) {
    sl.h_table[k] = job_trace(frames[k].scene, frames[k].fb, frames[k].W * frames[k].H);
    ok[k]->batch = nj;
  }
  auto encode = [&]() {
    if (batched) {
      cudaMemcpyAsync(sl.d_table, sl.h_table, sizeof(JobTrace) * nj, cudaMemcpyHostToDevice, sl.stream);
      encode_batch_plain(frames, nj, cfg, sl.d_table, s->num_sms, sl.stream);
    } else {
      const BatchFrame& f = frames[0];
      encode_frame(f.scene, f.fb, cfg, f.mats, f.W, f.H, f.frame_idx, s->num_sms, sl.stream, nullptr);
    }
    for (int k = 0; k < nj; ++k) {
      Job* j = ok[k];
      float* dst = j->out_pinned ? j->out : j->staging;
      cudaMemcpyAsync(dst, frames[k].fb.out_rgb, (size_t)frames[k].W * frames[k].H * 12, cudaMemcpyDeviceToHost,
                      sl.stream);
    }
  };
  cudaError_t e = cudaSuccess;
  int mode = 0;
  cudaEventRecord(sl.ev0, sl.stream);
  if (s->use_graphs) {
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(sl.stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      encode();
      e = cudaStreamEndCapture(sl.stream, &g);
    }
    if (e == cudaSuccess) {
      cudaGraphExec_t& exec = sl.execs[shape_key(cfg, nj)];
      cudaGraphExecUpdateResultInfo info;
      if (exec && cudaGraphExecUpdate(exec, g, &info) == cudaSuccess) {
        mode = 2;
        s->graph_updates++;
      } else {
        cudaGetLastError();  // a failed update leaves a recoverable error
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        e = cudaGraphInstantiate(&exec, g, 0);
        mode = 1;
        s->graph_instantiations++;
      }
      cudaGraphDestroy(g);
      if (e == cudaSuccess) e = cudaGraphLaunch(exec, sl.stream);
    }
  } else {
    encode();
    e = cudaGetLastError();
  }
  cudaEventRecord(sl.ev1, sl.stream);
  for (Job* j : ok) {
    j->graph_mode = mode;
    if (e != cudaSuccess) {
      j->rc = AP_E_CUDA;
      j->err = std::string("job launch: ") + cudaGetErrorString(e);
    }
  }
  cudaLaunchHostFunc(sl.stream, on_slot_done, new CallbackArg{s, (int)(&sl - &s->slots[0])});
  return true;
}

void dispatcher(Server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    // completions
    for (size_t i = 0; i < s->slots.size(); ++i) {
      Slot& sl = s->slots[i];
      if (sl.jobs.empty() || !sl.finished) continue;
      cudaError_t e = cudaEventSynchronize(sl.ev1);  // already complete: returns at once
      float ms = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, sl.ev0, sl.ev1);
      for (size_t k = 0; k < sl.jobs.size(); ++k) {
        Job* j = sl.jobs[k];
        if (e != cudaSuccess && j->rc == AP_OK) {
          j->rc = AP_E_CUDA;
          j->err = std::string("job: ") + cudaGetErrorString(e);
        }
        if (j->rc == AP_OK && j->cancelled) {
          j->rc = AP_E_CANCELLED;
          j->err = "job cancelled while it ran";
        }
        if (j->rc == AP_OK && !j->out_pinned)
          std::memcpy(j->out, j->staging, (size_t)j->desc.width * j->desc.height * 12);
        if (j->dev) cudaFreeAsync(j->dev, sl.stream);
        j->dev = nullptr;
        s->in_use -= j->bytes;
        j->gpu_ms = ms;
        j->t_done = Clock::now();
        j->done = true;
        s->completed++;
      }
      sl.jobs.clear();
      sl.finished = false;
      s->cv_done.notify_all();
    }
    // queued jobs past their deadline complete without running
    const Clock::time_point now = Clock::now();
    for (auto it = s->pending.begin(); it != s->pending.end();) {
      Job* j = *it;
      if (j->desc.deadline_ms && ms_between(j->t_submit, now) >= (double)j->desc.deadline_ms) {
        j->rc = AP_E_TIMEOUT;
        j->err = "job deadline passed in the queue";
        j->t_admit = j->t_done = now;
        j->done = true;
        s->completed++;
        it = s->pending.erase(it);
        s->cv_done.notify_all();
      } else {
        ++it;
      }
    }
    // admissions, in arrival order; a batch takes the head job and the later
    // queued jobs of the same shape that fit the budget
    while (!s->pending.empty()) {
      int free_slot = -1;
      for (size_t i = 0; i < s->slots.size(); ++i)
        if (s->slots[i].jobs.empty()) {
          free_slot = (int)i;
          break;
        }
      if (free_slot < 0) break;
      Job* j = s->pending.front();
      if (s->scene_bytes + s->in_use + j->bytes > s->budget) {
        if (s->in_use == 0) {  // cannot fit even alone
          s->pending.pop_front();
          j->rc = AP_E_OOM;
          j->err = "job frame state exceeds the device-memory budget";
          j->t_admit = j->t_done = Clock::now();
          j->done = true;
          s->completed++;
          s->cv_done.notify_all();
          continue;
        }
        break;  // wait for memory to free up
      }
      s->pending.pop_front();
      std::vector<Job*> batch{j};
      size_t bytes = j->bytes;
      if (batchable(s->base) && s->max_batch > 1) {
        for (auto it = s->pending.begin(); it != s->pending.end() && batch.size() < s->max_batch;) {
          Job* o = *it;
          if (same_shape(o->desc, j->desc) && s->scene_bytes + s->in_use + bytes + o->bytes <= s->budget) {
            batch.push_back(o);
            bytes += o->bytes;
            it = s->pending.erase(it);
          } else {
            ++it;
          }
        }
      }
      Slot& sl = s->slots[free_slot];
      std::vector<Job*> admitted;
      for (size_t k = 0; k < batch.size(); ++k) {
        Job* b = batch[k];
        const size_t out_bytes = (size_t)b->desc.width * b->desc.height * 12;
        if (!b->out_pinned && sl.staging_bytes[k] < out_bytes) {
          lk.unlock();
          if (sl.staging[k]) cudaFreeHost(sl.staging[k]);
          sl.staging[k] = nullptr;
          cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&sl.staging[k]), out_bytes, cudaHostAllocDefault);
          lk.lock();
          sl.staging_bytes[k] = e == cudaSuccess ? out_bytes : 0;
          if (e != cudaSuccess) {
            sl.staging[k] = nullptr;
            b->rc = AP_E_OOM;
            b->err = "pinned staging buffer";
            b->t_admit = b->t_done = Clock::now();
            b->done = true;
            s->completed++;
            s->cv_done.notify_all();
            continue;
          }
        }
        b->staging = sl.staging[k];  // buffer k of the slot is this job's alone
        admitted.push_back(b);
      }
      if (admitted.empty()) continue;
      const std::vector<Job*>& launched = admitted;
      const Clock::time_point t_admit = Clock::now();
      for (Job* b : launched) {
        b->slot = free_slot;
        b->t_admit = t_admit;
        s->in_use += b->bytes;
      }
      s->peak = std::max(s->peak, s->scene_bytes + s->in_use);
      sl.jobs = launched;
      sl.finished = false;
      lk.unlock();
      std::vector<Job*> enq, failed;
      const bool enqueued = launch_batch(s, sl, launched, &enq, &failed);
      lk.lock();
      sl.jobs = enq;
      for (Job* b : failed) {
        s->in_use -= b->bytes;
        b->t_done = Clock::now();
        b->done = true;
        s->completed++;
      }
      if (!enqueued) sl.jobs.clear();
      if (!failed.empty() || !enqueued) s->cv_done.notify_all();
    }
    bool inflight = false;
    for (const Slot& sl : s->slots) inflight = inflight || !sl.jobs.empty();
    if (s->stop && s->pending.empty() && !inflight) break;
    bool ready = false;
    for (const Slot& sl : s->slots) ready = ready || (!sl.jobs.empty() && sl.finished);
    if (!ready) {
      // sleep until a completion, a submission, or the nearest queued deadline
      double wait_ms = -1.0;
      for (const Job* j : s->pending)
        if (j->desc.deadline_ms) {
          const double left = (double)j->desc.deadline_ms - ms_between(j->t_submit, Clock::now());
          wait_ms = wait_ms < 0.0 ? left : std::min(wait_ms, left);
        }
      if (wait_ms < 0.0) s->cv_work.wait(lk);
      else if (wait_ms > 0.0) s->cv_work.wait_for(lk, std::chrono::duration<double, std::milli>(wait_ms));
    }
  }
}

int srv_fail(Server* s, int code, const std::string& msg) {
  if (s) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = msg;
  }
  return code;
}

}  // namespace

extern "C" {

void* ap_server_create(const ap_frame_config* cfg, int device, uint64_t hbm_budget, uint32_t max_inflight,
                       int use_graphs, int* err) {
  if (err) *err = AP_OK;
  if (!cfg || max_inflight == 0 || max_inflight > 64 || hbm_budget == 0) {
    if (err) *err = AP_E_INVALID;
    return nullptr;
  }
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    if (err) *err = AP_E_CUDA;
    return nullptr;
  }
  ap::DeviceScope device_scope(device);
  Server* s = new Server;
  s->device = device;
  s->budget = hbm_budget;
  s->use_graphs = use_graphs;
  std::memcpy(&s->base, cfg, sizeof(FrameConfig));
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
  // The server's own pool, so that job state freed between jobs stays mapped
  // for the next job (no release back to the driver) without changing the
  // device's default pool, which belongs to the whole process.
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  bool ok = cudaMemPoolCreate(&s->pool, &props) == cudaSuccess;
  if (ok) {
    uint64_t thr = UINT64_MAX;
    ok = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr) == cudaSuccess;
  }
  s->slots.resize(max_inflight);
  for (Slot& sl : s->slots) {
    if (!ok) break;
    ok = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreate(&sl.ev0) == cudaSuccess && cudaEventCreate(&sl.ev1) == cudaSuccess &&
         cudaHostAlloc(reinterpret_cast<void**>(&sl.h_table), sizeof(JobTrace) * kMaxBatch, cudaHostAllocDefault) ==
             cudaSuccess &&
         cudaMalloc(&sl.d_table, sizeof(JobTrace) * kMaxBatch) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    if (err) *err = AP_E_CUDA;
    for (Slot& t : s->slots) {
      if (t.stream) cudaStreamDestroy(t.stream);
      if (t.ev0) cudaEventDestroy(t.ev0);
      if (t.ev1) cudaEventDestroy(t.ev1);
      if (t.h_table) cudaFreeHost(t.h_table);
      if (t.d_table) cudaFree(t.d_table);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return nullptr;
  }
  s->worker = std::thread(dispatcher, s);
  return s;
}

void ap_server_destroy(void* sp) {
  Server* s = static_cast<Server*>(sp);
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();  // drains queued and in-flight jobs
  ap::DeviceScope device_scope(s->device);
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    for (auto& kv : sl.execs)
      if (kv.second) cudaGraphExecDestroy(kv.second);
    sl.execs.clear();
    for (float* p : sl.staging)
      if (p) cudaFreeHost(p);
    if (sl.h_table) cudaFreeHost(sl.h_table);
    if (sl.d_table) cudaFree(sl.d_table);
    if (sl.ev0) cudaEventDestroy(sl.ev0);
    if (sl.ev1) cudaEventDestroy(sl.ev1);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  for (auto& kv : s->jobs) delete kv.second;
  for (void* h : s->scenes) ap_destroy(h);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
}

const char* ap_server_last_error(const void* sp) {
  const Server* s = static_cast<const Server*>(sp);
  return s ? s->err.c_str() : "null server";
}

int ap_server_add_scene(void* sp, const ap_scene_desc* desc, uint32_t* scene_id) {
  Server* s = static_cast<Server*>(sp);
  if (!s || !desc || !scene_id) return AP_E_INVALID;
  int e = 0;
  void* h = ap_create(reinterpret_cast<const ap_frame_config*>(&s->base), s->device, &e);
  if (!h) return srv_fail(s, e ? e : AP_E_CUDA, "scene handle");
  int rc = ap_scene_upload(h, desc);
  if (rc != AP_OK) {
    std::string msg = ap_last_error(h);
    ap_destroy(h);
    return srv_fail(s, rc, "scene upload: " + msg);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->scenes.push_back(h);
  s->scene_bytes += ap::handle_scene_bytes(h);
  *scene_id = (uint32_t)(s->scenes.size() - 1);
  return AP_OK;
}

uint64_t ap_server_job_bytes(uint32_t width, uint32_t height) { return frame_buffer_bytes(width, height); }

int ap_server_submit(void* sp, const ap_job* job, float* out_rgb, size_t out_bytes, uint64_t* ticket) {
  Server* s = static_cast<Server*>(sp);
  if (!s || !job || !out_rgb || !ticket) return AP_E_INVALID;
  if (job->width == 0 || job->height == 0 || (uint64_t)job->width * job->height > (1ull << 26))
    return srv_fail(s, AP_E_INVALID, "job: bad resolution");
  if (job->spp == 0 || job->spp > 4096 || job->max_depth == 0 || job->max_depth > 64)
    return srv_fail(s, AP_E_INVALID, "job: spp or depth out of range");
  if (out_bytes < (size_t)job->width * job->height * 12) return srv_fail(s, AP_E_INVALID, "job: output buffer too small");
  cudaPointerAttributes attr;
  bool pinned = cudaPointerGetAttributes(&attr, out_rgb) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  Job* j = new Job;
  j->desc = *job;
  j->out = out_rgb;
  j->out_pinned = pinned;
  j->bytes = frame_buffer_bytes(job->width, job->height);
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (job->scene >= s->scenes.size()) {
      delete j;
      s->err = "job: unknown scene";
      return AP_E_INVALID;
    }
    j->ticket = s->next_ticket++;
    s->jobs[j->ticket] = j;
    s->pending.push_back(j);
    *ticket = j->ticket;
  }
  s->cv_work.notify_one();
  return AP_OK;
}

int ap_server_query(void* sp, uint64_t ticket, int* done) {
  Server* s = static_cast<Server*>(sp);
  if (!s || !done) return AP_E_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return AP_E_INVALID;
  *done = it->second->done ? 1 : 0;
  return AP_OK;
}

int ap_server_wait(void* sp, uint64_t ticket, ap_job_result* res) {
  Server* s = static_cast<Server*>(sp);
  if (!s) return AP_E_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) {
    s->err = "unknown ticket";
    return AP_E_INVALID;
  }
  Job* j = it->second;
  s->cv_done.wait(lk, [&] { return j->done; });
  if (res) {
    res->queued_ms = ms_between(j->t_submit, j->t_admit);
    res->total_ms = ms_between(j->t_submit, j->t_done);
    res->gpu_ms = j->gpu_ms;
    res->device_bytes = j->bytes;
    res->graph_mode = (uint32_t)j->graph_mode;
    res->slot = (uint32_t)j->slot;
    res->batch = (uint32_t)j->batch;
    res->pad = 0;
  }
  int rc = j->rc;
  if (rc != AP_OK) s->err = j->err;
  s->jobs.erase(it);
  delete j;
  return rc;
}

int ap_server_cancel(void* sp, uint64_t ticket) {
  Server* s = static_cast<Server*>(sp);
  if (!s) return AP_E_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) {
      s->err = "unknown ticket";
      return AP_E_INVALID;
    }
    Job* j = it->second;
    if (j->done) return AP_OK;
    auto q = std::find(s->pending.begin(), s->pending.end(), j);
    if (q != s->pending.end()) {  // still queued: dropped
      s->pending.erase(q);
      j->rc = AP_E_CANCELLED;
      j->err = "job cancelled before it started";
      j->t_admit = j->t_done = Clock::now();
      j->done = true;
      s->completed++;
      s->cv_done.notify_all();
    } else {
      j->cancelled = true;  // on the GPU: reported when its launches finish
    }
  }
  s->cv_work.notify_one();
  return AP_OK;
}

int ap_server_set_batching(void* sp, uint32_t max_batch) {
  Server* s = static_cast<Server*>(sp);
  if (!s || max_batch == 0 || max_batch > (uint32_t)kMaxBatch) return AP_E_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->max_batch = max_batch;
  }
  s->cv_work.notify_one();
  return AP_OK;
}

int ap_server_stats(void* sp, uint64_t* out8) {
  Server* s = static_cast<Server*>(sp);
  if (!s || !out8) return AP_E_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  uint64_t inflight = 0;
  for (const Slot& sl : s->slots) inflight += sl.jobs.size();
  out8[0] = s->completed;
  out8[1] = inflight;
  out8[2] = s->pending.size();
  out8[3] = s->scene_bytes + s->in_use;
  out8[4] = s->peak;
  out8[5] = s->scene_bytes;
  out8[6] = s->graph_instantiations.load();
  out8[7] = s->graph_updates.load();
  return AP_OK;
}

}  // extern "C"
