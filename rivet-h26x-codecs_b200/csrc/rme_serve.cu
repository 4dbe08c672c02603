// The serving loop: per-frame ME requests from many streams, searched as
// they arrive. A frame is uploaded into its stream's ring of resident
// pictures on the upload stream; streams are admitted against an HBM budget
// of their resident pictures. Two modes:
//
//   RME_SERVE_LAUNCHES: the frames admitted since the last launch go into
//   one search launch of their own as soon as one of kLaunchStreams launch
//   streams is free, so launches overlap on the device (a frame that
//   arrives while others are searched starts at once on another stream); a
//   launch of one or two 1080p frames runs the latency form (the row form
//   for HEVC), a larger one the throughput form.
//
//   RME_SERVE_RESIDENT: frames join the resident engine's running search
//   (rme_engine.cu) behind their uploads, as soon as a frame slot and ring
//   room are free; their work shares the SMs with the frames already in
//   flight.
//
// One worker thread owns the context: it admits requests, launches or
// submits them, polls for finished searches (launch events, or the
// engine's completion flags in host memory the device writes), copies
// finished frames' results out on a copy stream and posts the completions.
// Frames are searched STANDALONE against the stream's previous `nref`
// source pictures (the reference's ME stage as a pre-pass, without the
// reconstruction loop).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "rme_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

// Frames of one stream in flight at once: its picture ring holds nref +
// kPerStream pictures, and a picture is refilled only once every frame that
// reads it is complete.
constexpr int kPerStream = 4;

struct Stream {
  rme_picture_desc d{};
  rme_params p{};
  int nref = 0;
  int64_t frames = 0;        // frames admitted so far
  uint64_t bytes = 0;        // resident bytes charged against the budget
  bool closing = false;
  int pending = 0;           // requests queued or in flight
  int32_t pic_base = 0;      // picture ids pic_base .. pic_base + nref + kPerStream - 1
  std::set<int64_t> open;    // frame numbers admitted and not yet complete
};

struct Request {
  int64_t id = 0;
  int32_t stream = 0;
  void* luma = nullptr;      // pinned copy of the frame (from the pool)
  size_t bytes = 0;
  rme_result* out = nullptr;
  bool out_pinned = false;   // results go straight into `out`
  double submit_s = 0.0;
  // in flight
  int64_t frame = -1;        // the stream's frame number
  int slot = -1;             // the engine's frame slot, or the launch stream (-1: not searched)
  int nresults = 0;
  rme_result* staging = nullptr;
  size_t staging_n = 0;
  cudaEvent_t ev = nullptr;  // the upload (first frames) or the results copy
  int status = 0;
  double t_start = 0.0, t_flag = 0.0;  // host clock: handed to the engine, its flag seen
  int64_t offset = 0;        // launch mode: the first result's index in the launch's buffer
};

// Launch mode: one of the launch streams, with the launch in flight on it.
constexpr int kLaunchStreams = 3;
struct LaunchStream {
  cudaStream_t s = nullptr;
  cudaEvent_t up = nullptr, done = nullptr, copied = nullptr;
  rme_result* d_out = nullptr;  // the launch's results (device memory)
  size_t cap = 0;
  bool busy = false;
  std::vector<Request> reqs;    // the frames it searches
};

struct Server {
  void* ctx = nullptr;
  int device = 0;
  rme_serve_opts o{};
  Clock::time_point t0 = Clock::now();
  std::mutex m;
  std::condition_variable cv;
  std::deque<Request> queue;
  std::vector<rme_completion> done;
  std::map<int32_t, Stream> streams;
  uint64_t resident = 0;
  int64_t next_id = 0;
  int32_t next_pic_base = 1 << 20;
  bool stop = false;
  int closes = 0;  // close_stream calls the worker has not yet looked at
  std::thread worker;
  // Pinned frame buffers by size: a submit copies into one, the upload reads
  // it asynchronously, the worker returns it once its frame is complete.
  std::map<size_t, std::vector<void*>> pool;
  // worker-only state
  bool resident_engine = false;  // RME_SERVE_RESIDENT
  rme::Engine* eng = nullptr;
  LaunchStream ls[kLaunchStreams];
  std::deque<Request> unlaunched;  // launch mode: admitted, waiting for a free launch stream
  cudaStream_t upload = nullptr, copy = nullptr;
  uint32_t* h_status = nullptr;  // pinned: the engine's status word, read back with each copy
  std::vector<Request> searching, copying, submitting;
  std::vector<cudaEvent_t> events;
  std::map<size_t, std::vector<rme_result*>> staging_pool;
  std::vector<std::pair<int32_t, int>> release_later;  // closed streams' pictures (id base, count)
  bool trace = false;  // RME_SERVE_TRACE=1: one line per frame on stderr
  double idle_since = 0.0;  // nothing in flight since

  void* take_buffer(size_t bytes) {  // lock held; null when the pool has none of this size
    auto& v = pool[bytes];
    if (v.empty()) return nullptr;
    void* b = v.back();
    v.pop_back();
    return b;
  }
  cudaEvent_t take_event() {
    if (!events.empty()) {
      cudaEvent_t e = events.back();
      events.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
  }
  rme_result* take_staging(size_t n) {
    auto& v = staging_pool[n];
    if (!v.empty()) {
      rme_result* b = v.back();
      v.pop_back();
      return b;
    }
    void* b = nullptr;
    return cudaMallocHost(&b, std::max<size_t>(n, 1) * sizeof(rme_result)) == cudaSuccess ? (rme_result*)b : nullptr;
  }

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
  void admit(std::vector<Request>& taken);
  rme_frame frame_of(const Stream& st, int64_t j) const;
  void submit_search(Request& r, const Stream& st);
  void start(Request& r);
  void launch_batch(LaunchStream& L, int k);
  void poll_launches();
  void finish(Request& r, double t);
  void release_closed(bool engine_idle);
};

// Device bytes of one resident picture of this format: the padded planes
// (16 for HEVC, 4 for H.264, rows padded to 128 bytes), as uploads lay them
// out.
uint64_t picture_bytes(const rme_picture_desc& d) {
  const bool h264 = d.codec == RME_CODEC_H264;
  const int cw = h264 ? (d.width + 15) / 16 * 16 : d.width, ch = h264 ? (d.height + 15) / 16 * 16 : d.height;
  const int pad = h264 ? rme::kH264Pad : rme::kHevcPad, bps = d.bit_depth == 8 ? 1 : 2;
  const uint64_t stride_bytes = ((uint64_t)(cw + 2 * pad) * bps + 127) / 128 * 128;
  return stride_bytes * (uint64_t)(ch + 2 * pad) * (h264 ? 4 : 16) + 256;
}

// Requests that may start now, oldest first (lock held): a stream's frame
// waits while the frame kPerStream before it is incomplete (its picture
// slot would be refilled under a search), and a stream's frames keep their
// order.
void Server::admit(std::vector<Request>& taken) {
  std::set<int32_t> blocked;
  for (auto it = queue.begin(); it != queue.end();) {
    Stream& st = streams[it->stream];
    const int64_t j = st.frames;
    const bool room = st.open.empty() || *st.open.begin() > j - kPerStream;
    if (blocked.count(it->stream) || !room) {
      blocked.insert(it->stream);
      ++it;
      continue;
    }
    it->frame = j;
    ++st.frames;
    st.open.insert(j);
    taken.push_back(std::move(*it));
    it = queue.erase(it);
  }
}

// Frame j of a stream: its picture slot and its references' (the previous
// nref pictures of the ring).
rme_frame Server::frame_of(const Stream& st, int64_t j) const {
  const int slots = st.nref + kPerStream;
  rme_frame f{};
  f.src_id = st.pic_base + (int32_t)(j % slots);
  f.nref = (int)std::min<int64_t>(st.nref, j);
  for (int k = 0; k < f.nref; ++k) f.ref_ids[k] = st.pic_base + (int32_t)((j - 1 - k) % slots);
  return f;
}

// Hand a frame (uploaded) to the engine; without room there, try again
// when a frame finishes; on an error, complete it behind its upload.
void Server::submit_search(Request& r, const Stream& st) {
  const rme_frame f = frame_of(st, r.frame);
  const int rc = rme::engine_submit(eng, &f, &st.p, upload, &r.slot);
  if (rc == RME_EBUSY) {
    r.slot = -1;
    submitting.push_back(r);
    return;
  }
  if (rc == 0) {
    r.nresults = rme::engine_slot_tasks(eng, r.slot);
    searching.push_back(r);
    return;
  }
  r.status = rc;
  r.slot = -1;
  r.ev = take_event();
  cudaEventRecord(r.ev, upload);
  copying.push_back(r);
}

// Upload the frame into its stream's ring, then (frames with a reference)
// submit it to the engine behind the upload.
void Server::start(Request& r) {
  r.t_start = now();
  const Stream* st;
  {
    std::lock_guard<std::mutex> lk(m);
    st = &streams[r.stream];
  }
  const rme_frame f = frame_of(*st, r.frame);
  // The picture's own search reads only its integer plane: it is handed to
  // the engine before the interpolated planes, which only later frames
  // read, are built behind it on the same stream.
  r.status = rme::ctx_picture_upload(ctx, f.src_id, &st->d, r.luma, 1, false, upload);
  if (r.status == 0 && f.nref > 0) {
    const size_t ns = searching.size(), nb = submitting.size(), nc = copying.size();
    submit_search(r, *st);  // the request goes into one of the three lists
    const int rc = rme_picture_build_planes(ctx, f.src_id, upload);
    Request* q = searching.size() > ns ? &searching.back()
                 : submitting.size() > nb ? &submitting.back()
                 : copying.size() > nc ? &copying.back()
                                       : nullptr;
    if (rc != 0 && q && q->status == 0) q->status = rc;
    return;
  }
  if (r.status == 0) r.status = rme_picture_build_planes(ctx, f.src_id, upload);
  // Not searched (a stream's first frame) or failed: complete once the
  // upload has read the frame's buffer.
  r.slot = -1;
  r.ev = take_event();
  cudaEventRecord(r.ev, upload);
  copying.push_back(r);
}

// Launch mode: the oldest admitted frames (at most max_frames_per_launch)
// go into one launch on launch stream k. Each is uploaded into its stream's
// ring on the upload stream; its interpolated planes are built there before
// the launch only when a later frame of the same launch reads it, else
// behind the launch's wait (they run beside the search: only later frames
// read them). The launch waits for the uploads and for the copies out of its
// buffer from the stream's previous launch; its results stay in device
// memory until poll_launches copies each frame's out.
void Server::launch_batch(LaunchStream& L, int k) {
  std::vector<Request> batch;
  while (!unlaunched.empty() && (int)batch.size() < o.max_frames_per_launch) {
    batch.push_back(std::move(unlaunched.front()));
    unlaunched.pop_front();
  }
  std::map<int32_t, size_t> last;  // a stream's last frame in the batch
  for (size_t i = 0; i < batch.size(); ++i) last[batch[i].stream] = i;
  std::vector<rme_frame> frames;
  std::vector<rme_params> params;
  std::vector<int64_t> offs;
  std::vector<size_t> searched;
  std::vector<int32_t> planes_after;
  int64_t total = 0;
  for (size_t i = 0; i < batch.size(); ++i) {
    Request& r = batch[i];
    r.t_start = now();
    const Stream* st;
    {
      std::lock_guard<std::mutex> lk(m);
      st = &streams[r.stream];
    }
    const rme_frame f = frame_of(*st, r.frame);
    const bool read_here = last[r.stream] != i;
    r.status = rme::ctx_picture_upload(ctx, f.src_id, &st->d, r.luma, 1, read_here, upload);
    if (r.status == 0 && !read_here) planes_after.push_back(f.src_id);
    int32_t cnt = 0;
    if (r.status == 0 && f.nref > 0) r.status = rme_frame_result_count(ctx, &f, &st->p, &cnt);
    if (r.status != 0 || f.nref == 0) {
      // Not searched (a stream's first frame) or failed: complete once the
      // upload has read the frame's buffer.
      r.slot = -1;
      r.ev = take_event();
      cudaEventRecord(r.ev, upload);
      copying.push_back(r);
      continue;
    }
    r.offset = total;
    r.nresults = cnt;
    total += cnt;
    frames.push_back(f);
    params.push_back(st->p);
    offs.push_back(r.offset);
    searched.push_back(i);
  }
  if (!frames.empty()) {
    int rc = 0;
    if (L.cap < (size_t)total) {
      if (L.d_out) {
        cudaEventSynchronize(L.copied);
        cudaFree(L.d_out);
      }
      L.d_out = nullptr;
      L.cap = 0;
      if (cudaMalloc(&L.d_out, sizeof(rme_result) * total) == cudaSuccess) L.cap = (size_t)total;
      else rc = RME_ENOMEM;
    }
    if (rc == 0 && (cudaEventRecord(L.up, upload) != cudaSuccess || cudaStreamWaitEvent(L.s, L.up, 0) != cudaSuccess ||
                    cudaStreamWaitEvent(L.s, L.copied, 0) != cudaSuccess))
      rc = RME_ECUDA;
    if (rc == 0)
      rc = rme_batch_search_async(ctx, frames.data(), params.data(), (int32_t)frames.size(), L.d_out, offs.data(), L.s);
    if (rc == 0 && cudaEventRecord(L.done, L.s) != cudaSuccess) rc = RME_ECUDA;
    for (size_t j : searched) {
      Request& r = batch[j];
      if (rc != 0) {
        r.status = rc;
        r.slot = -1;
        r.ev = take_event();
        cudaEventRecord(r.ev, upload);
        copying.push_back(r);
      } else {
        r.slot = k;
        L.reqs.push_back(r);
      }
    }
    L.busy = !L.reqs.empty();
  }
  for (int32_t id : planes_after) rme_picture_build_planes(ctx, id, upload);
}

// Launch mode: finished launches (their event) are completed on the
// context (status, launch slot), and each frame's results are copied out
// on the copy stream into the caller's buffer (pinned) or a staging one.
void Server::poll_launches() {
  for (LaunchStream& L : ls) {
    if (!L.busy || cudaEventQuery(L.done) != cudaSuccess) continue;
    cudaGetLastError();
    uint32_t dev_status = 0;
    const int rc = rme_sync(ctx, L.s, &dev_status);
    const double t = now();
    for (Request& r : L.reqs) {
      r.t_flag = t;
      if (rc != 0) r.status = rc;
      rme_result* dst = r.out;
      if (!r.out_pinned) {
        r.staging = take_staging((size_t)r.nresults);
        r.staging_n = (size_t)r.nresults;
        dst = r.staging;
      }
      if (r.status == 0 &&
          (!dst || cudaMemcpyAsync(dst, L.d_out + r.offset, sizeof(rme_result) * r.nresults, cudaMemcpyDeviceToHost,
                                   copy) != cudaSuccess))
        r.status = RME_ECUDA;
      r.ev = take_event();
      cudaEventRecord(r.ev, copy);
      copying.push_back(r);
    }
    cudaEventRecord(L.copied, copy);
    L.reqs.clear();
    L.busy = false;
  }
}

void Server::finish(Request& r, double t) {  // lock held
  rme_completion c{};
  c.request_id = r.id;
  c.stream_id = r.stream;
  c.status = r.status;
  c.submit_s = r.submit_s;
  c.done_s = t;
  c.nresults = r.status == 0 && r.slot >= 0 ? r.nresults : 0;
  done.push_back(c);
  pool[r.bytes].push_back(r.luma);
  Stream& st = streams[r.stream];
  st.open.erase(r.frame);
  --st.pending;
}

// Drop closed streams with nothing queued or in flight (their budget is
// free at once); their pictures are released while no engine kernel runs (a
// device free waits for every kernel).
void Server::release_closed(bool engine_idle) {
  std::vector<std::pair<int32_t, int>> now;
  {
    std::lock_guard<std::mutex> lk(m);
    for (auto it = streams.begin(); it != streams.end();) {
      if (it->second.closing && it->second.pending == 0) {
        release_later.emplace_back(it->second.pic_base, it->second.nref + kPerStream);
        resident -= it->second.bytes;
        it = streams.erase(it);
      } else {
        ++it;
      }
    }
    if (engine_idle) now.swap(release_later);
  }
  for (auto& pr : now)
    for (int k = 0; k < pr.second; ++k) rme_picture_release(ctx, pr.first + k);
}

void Server::run() {
  for (;;) {
    std::vector<Request> taken;
    bool any_close = false;
    bool launches_busy = !unlaunched.empty();
    for (const LaunchStream& L : ls) launches_busy |= L.busy;
    const bool busy = !searching.empty() || !copying.empty() || !submitting.empty() || launches_busy;
    {
      std::unique_lock<std::mutex> lk(m);
      if (busy)
        cv.wait_for(lk, std::chrono::microseconds(20), [&] { return stop || !queue.empty() || closes > 0; });
      else
        cv.wait_for(lk, std::chrono::milliseconds(50),
                    [&] { return stop || !queue.empty() || closes > 0 || !release_later.empty(); });
      if (stop && queue.empty() && !busy) break;
      any_close = closes > 0;
      closes = 0;
      admit(taken);
    }
    if (resident_engine) {
      for (Request& r : taken) start(r);
    } else {
      for (Request& r : taken) unlaunched.push_back(std::move(r));
      poll_launches();
      for (int k = 0; k < kLaunchStreams && !unlaunched.empty(); ++k)
        if (!ls[k].busy) launch_batch(ls[k], k);
    }
    // Frames the engine had no room for: again, oldest first.
    if (!submitting.empty()) {
      std::vector<Request> again;
      again.swap(submitting);
      for (Request& r : again) {
        const Stream* st;
        {
          std::lock_guard<std::mutex> lk(m);
          st = &streams[r.stream];
        }
        submit_search(r, *st);
      }
    }
    // Finished searches: their results out on the copy stream.
    for (size_t i = 0; i < searching.size();) {
      Request& r = searching[i];
      if (!rme::engine_done(eng, r.slot)) {
        ++i;
        continue;
      }
      r.t_flag = now();
      rme_result* dst = r.out;
      if (!r.out_pinned) {
        r.staging = take_staging((size_t)r.nresults);
        r.staging_n = (size_t)r.nresults;
        dst = r.staging;
      }
      cudaError_t e = dst ? cudaMemcpyAsync(dst, rme::engine_results(eng, r.slot), sizeof(rme_result) * r.nresults,
                                            cudaMemcpyDeviceToHost, copy)
                          : cudaErrorMemoryAllocation;
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_status, rme::engine_status_word(eng), sizeof(uint32_t), cudaMemcpyDeviceToHost, copy);
      r.ev = take_event();
      cudaEventRecord(r.ev, copy);
      if (e != cudaSuccess) r.status = RME_ECUDA;
      copying.push_back(r);
      searching[i] = searching.back();
      searching.pop_back();
    }
    // The engine leaves when idle: launch it again while frames are in flight.
    if (resident_engine && !searching.empty()) rme::engine_keep_running(eng);
    // Copies done: results to the caller, slots back to the engine.
    bool any = false;
    for (size_t i = 0; i < copying.size();) {
      Request& r = copying[i];
      if (cudaEventQuery(r.ev) != cudaSuccess) {
        ++i;
        continue;
      }
      if (r.slot >= 0) {
        if (resident_engine && r.status == 0 && *(volatile uint32_t*)h_status != 0) r.status = RME_EDEVICE;
        if (r.status == 0 && r.staging) std::memcpy(r.out, r.staging, sizeof(rme_result) * r.nresults);
        if (resident_engine) rme::engine_release(eng, r.slot);
      }
      if (r.staging) staging_pool[r.staging_n].push_back(r.staging);
      events.push_back(r.ev);
      const double t = now();
      if (trace)
        std::fprintf(stderr, "serve: stream %d frame %lld slot %d: queued %.3f ms, engine %.3f ms, copy %.3f ms\n",
                     r.stream, (long long)r.frame, r.slot, (r.t_start - r.submit_s) * 1e3,
                     r.slot >= 0 ? (r.t_flag - r.t_start) * 1e3 : 0.0, r.slot >= 0 ? (t - r.t_flag) * 1e3 : 0.0);
      {
        std::lock_guard<std::mutex> lk(m);
        finish(r, t);
      }
      any = true;
      copying[i] = copying.back();
      copying.pop_back();
    }
    // Nothing in flight for a while: stop the engine kernel (the waiting
    // warps leave), so that it holds no SM while the server is idle; the
    // next frame launches it again.
    if (!resident_engine) {
      bool in_flight = !unlaunched.empty();
      for (const LaunchStream& L : ls) in_flight |= L.busy;
      if (!release_later.empty() || any || any_close) release_closed(!in_flight);
      continue;
    }
    if (searching.empty() && submitting.empty()) {
      if (any || !taken.empty()) idle_since = now();
      else if (now() - idle_since > 0.02) rme::engine_stop(eng);
    } else {
      idle_since = now();
    }
    if (!release_later.empty() || any || any_close) release_closed(rme::engine_idle(eng));
  }
}

}  // namespace

extern "C" {

int rme_serve_start(void* ctx, const rme_serve_opts* o, void** server) {
  if (!ctx || !o || !server || o->max_frames_per_launch < 1 || o->max_frames_per_launch > 255 || o->max_streams < 1)
    return RME_EINVAL;
  if (o->mode != RME_SERVE_LAUNCHES && o->mode != RME_SERVE_RESIDENT) return RME_EINVAL;
  auto* s = new Server();
  s->ctx = ctx;
  s->o = *o;
  s->resident_engine = o->mode == RME_SERVE_RESIDENT;
  cudaGetDevice(&s->device);
  bool ok = true;
  // Launch mode: the searches' streams at the greatest priority and the
  // uploads' (whose plane builds run beside a search) at the least, so that
  // a search's blocks are placed before pending plane-build blocks.
  int prio_least = 0, prio_greatest = 0;
  cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (!s->resident_engine)
    for (LaunchStream& L : s->ls)
      ok = ok && cudaStreamCreateWithPriority(&L.s, cudaStreamNonBlocking, prio_greatest) == cudaSuccess &&
           cudaEventCreateWithFlags(&L.up, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&L.copied, cudaEventDisableTiming) == cudaSuccess;
  if (!ok || (s->resident_engine && rme::engine_create(ctx, s->device, &s->eng) != 0) ||
      cudaStreamCreateWithPriority(&s->upload, cudaStreamNonBlocking, s->resident_engine ? 0 : prio_least) !=
          cudaSuccess ||
      cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost(&s->h_status, 64) != cudaSuccess) {
    if (s->eng) rme::engine_destroy(s->eng);
    for (LaunchStream& L : s->ls) {
      for (cudaEvent_t e : {L.up, L.done, L.copied})
        if (e) cudaEventDestroy(e);
      if (L.s) cudaStreamDestroy(L.s);
    }
    if (s->upload) cudaStreamDestroy(s->upload);
    if (s->copy) cudaStreamDestroy(s->copy);
    if (s->h_status) cudaFreeHost(s->h_status);
    delete s;
    return RME_ECUDA;
  }
  *s->h_status = 0;
  s->trace = std::getenv("RME_SERVE_TRACE") && std::getenv("RME_SERVE_TRACE")[0] == '1';
  s->worker = std::thread([s] {
    cudaSetDevice(s->device);
    s->run();
  });
  *server = s;
  return RME_OK;
}

int rme_serve_open_stream(void* server, int32_t stream_id, const rme_picture_desc* d, const rme_params* p,
                          int32_t nref) {
  auto* s = (Server*)server;
  if (!s || !d || !p || nref < 1 || nref > RME_MAX_REFS || p->codec != d->codec ||
      p->predictor_mode != RME_PRED_STANDALONE)
    return RME_EINVAL;
  int32_t count = 0;
  // The format and settings are checked the way a search would check them.
  if (rme_standalone_blocks(d, p, nullptr, &count) != 0) return RME_EINVAL;
  const uint64_t bytes = picture_bytes(*d) * (uint64_t)(nref + kPerStream);
  // The stream's frame buffers (pinned host memory): as many as it can have
  // open at once, and two more, pinned here rather than on its first
  // submits, and before the lock (pinning is slow).
  const size_t fb = (size_t)d->stride * d->height * (d->bit_depth == 8 ? 1 : 2);
  std::vector<void*> bufs;
  for (int k = 0; k < kPerStream + 2; ++k) {
    void* b = nullptr;
    if (cudaMallocHost(&b, fb) != cudaSuccess) break;
    bufs.push_back(b);
  }
  std::lock_guard<std::mutex> lk(s->m);
  const int refuse = s->streams.count(stream_id) ? RME_EINVAL
                     : ((int)s->streams.size() >= s->o.max_streams || s->resident + bytes > s->o.hbm_budget_bytes)
                         ? RME_EBUSY
                         : 0;
  if (refuse) {
    for (void* b : bufs) cudaFreeHost(b);
    return refuse;
  }
  Stream st;
  st.d = *d;
  st.p = *p;
  st.nref = nref;
  st.bytes = bytes;
  st.pic_base = s->next_pic_base;
  s->next_pic_base += RME_MAX_REFS + kPerStream;
  s->resident += bytes;
  s->streams[stream_id] = st;
  for (void* b : bufs) s->pool[fb].push_back(b);
  return RME_OK;
}

int rme_serve_submit(void* server, int32_t stream_id, const void* luma, rme_result* out, int64_t* request_id) {
  auto* s = (Server*)server;
  if (!s || !luma) return RME_EINVAL;
  Request r;
  r.submit_s = s->now();
  if (out) {
    cudaPointerAttributes pa{};
    r.out_pinned = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
  }
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->streams.find(stream_id);
  if (it == s->streams.end() || it->second.closing) return RME_ENOTFOUND;
  const rme_picture_desc& d = it->second.d;
  r.bytes = (size_t)d.stride * d.height * (d.bit_depth == 8 ? 1 : 2);
  if ((it->second.frames > 0 || it->second.pending > 0) && !out) return RME_EINVAL;  // this frame is searched
  r.luma = s->take_buffer(r.bytes);
  if (!r.luma) {
    // Pinning host memory is slow: it is done without the lock, so the
    // worker and other submitters are not held up behind it.
    lk.unlock();
    if (cudaMallocHost(&r.luma, r.bytes) != cudaSuccess) return RME_ENOMEM;
    lk.lock();
    it = s->streams.find(stream_id);
    if (it == s->streams.end() || it->second.closing) {
      s->pool[r.bytes].push_back(r.luma);
      return RME_ENOTFOUND;
    }
  }
  r.id = ++s->next_id;
  r.stream = stream_id;
  r.out = out;
  ++it->second.pending;  // the stream stays open while its copy is made
  lk.unlock();
  std::memcpy(r.luma, luma, r.bytes);
  if (request_id) *request_id = r.id;
  lk.lock();
  s->queue.push_back(std::move(r));
  lk.unlock();
  s->cv.notify_one();
  return RME_OK;
}

int rme_serve_poll(void* server, rme_completion* done, int32_t max, int32_t* n) {
  auto* s = (Server*)server;
  if (!s || !n || max < 0 || (max > 0 && !done)) return RME_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  const int k = std::min<int>(max, (int)s->done.size());
  std::copy(s->done.begin(), s->done.begin() + k, done);
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return RME_OK;
}

int rme_serve_close_stream(void* server, int32_t stream_id) {
  auto* s = (Server*)server;
  if (!s) return RME_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->streams.find(stream_id);
    if (it == s->streams.end() || it->second.closing) return RME_ENOTFOUND;
    // The worker drops it once its last request completes.
    it->second.closing = true;
    ++s->closes;
  }
  s->cv.notify_one();
  return RME_OK;
}

int rme_serve_stop(void* server) {
  auto* s = (Server*)server;
  if (!s) return RME_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  rme::engine_destroy(s->eng);  // the kernel leaves (asked to), then its memory goes
  for (LaunchStream& L : s->ls) {
    if (L.s) cudaStreamSynchronize(L.s);
    if (L.d_out) cudaFree(L.d_out);
    for (cudaEvent_t e : {L.up, L.done, L.copied})
      if (e) cudaEventDestroy(e);
    if (L.s) cudaStreamDestroy(L.s);
  }
  for (auto& kv : s->streams)
    for (int k = 0; k < kv.second.nref + kPerStream; ++k) rme_picture_release(s->ctx, kv.second.pic_base + k);
  for (auto& pr : s->release_later)
    for (int k = 0; k < pr.second; ++k) rme_picture_release(s->ctx, pr.first + k);
  for (auto& q : s->queue) cudaFreeHost(q.luma);
  for (auto& kv : s->pool)
    for (void* b : kv.second) cudaFreeHost(b);
  for (auto& kv : s->staging_pool)
    for (rme_result* b : kv.second) cudaFreeHost(b);
  for (cudaEvent_t e : s->events) cudaEventDestroy(e);
  cudaFreeHost(s->h_status);
  cudaStreamDestroy(s->upload);
  cudaStreamDestroy(s->copy);
  delete s;
  return RME_OK;
}

}  // extern "C"
