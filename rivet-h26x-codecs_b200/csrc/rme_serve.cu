// The serving loop: a host thread that turns per-frame ME requests from many
// streams into batched persistent launches (continuous batching at launch
// granularity). Requests that arrive while a launch runs on the device wait
// in the queue and join the next launch; each stream keeps its reference
// pictures resident on the device, and streams are admitted against an HBM
// budget. It is a client of the library's own C ABI: uploads, the batched
// search, releases.
//
// Frames are searched STANDALONE against the stream's previous `nref`
// source pictures (the reference's ME stage run as a pre-pass, without the
// reconstruction loop), so a frame's references are ready as soon as they
// are uploaded. A stream contributes up to kPerStream frames (in order) to
// one launch; a copier thread moves finished results out while the next
// launch runs.
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
#include <thread>
#include <vector>

#include "rme_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Stream {
  rme_picture_desc d{};
  rme_params p{};
  int nref = 0;
  int64_t frames = 0;      // frames uploaded so far
  uint64_t bytes = 0;      // resident bytes charged against the budget
  bool closing = false;
  int pending = 0;         // requests queued or in flight
  int32_t pic_base = 0;    // picture ids pic_base .. pic_base + nref + kPerStream - 1
};

struct Request {
  int64_t id = 0;
  int32_t stream = 0;
  void* luma = nullptr;  // pinned copy of the frame (from the pool)
  size_t bytes = 0;
  rme_result* out = nullptr;
  double submit_s = 0.0;
};

// Frames of one stream that can join one launch (its picture ring holds
// nref + kPerStream pictures).
constexpr int kPerStream = 4;

// A launch handed from the worker to the copier.
struct Launch {
  std::vector<Request> batch;
  std::vector<int> status;
  std::vector<int64_t> offset, count;
  int slot = 0;
  size_t left = 0;
  double t_take = 0, t_up = 0, t_search = 0;
};

struct Server {
  void* ctx = nullptr;
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
  int cleanups = 0;  // closed streams whose pictures the worker must release
  std::thread worker;
  // Two pinned result buffers: the worker fills one while the copier
  // empties the other.
  rme_result* staging[2] = {nullptr, nullptr};
  size_t staging_n[2] = {0, 0};
  bool slot_busy[2] = {false, false};
  std::deque<Launch> copies;
  bool copier_stop = false;
  std::condition_variable copy_cv, copied_cv;
  // Pinned frame buffers by size: a submit copies into one, the upload reads
  // it asynchronously, the worker returns it once its launch is complete.
  std::map<size_t, std::vector<void*>> pool;

  void* take_buffer(size_t bytes) {  // lock held
    auto& v = pool[bytes];
    if (!v.empty()) {
      void* b = v.back();
      v.pop_back();
      return b;
    }
    void* b = nullptr;
    return cudaMallocHost(&b, bytes) == cudaSuccess ? b : nullptr;
  }

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
  void copy_loop();
  // Release the pictures of closed streams with nothing queued or in flight
  // (worker thread, lock held: only the worker touches the context).
  void release_closed() {
    for (auto it = streams.begin(); it != streams.end();) {
      if (it->second.closing && it->second.pending == 0) {
        for (int k = 0; k < it->second.nref + kPerStream; ++k) rme_picture_release(ctx, it->second.pic_base + k);
        resident -= it->second.bytes;
        it = streams.erase(it);
      } else {
        ++it;
      }
    }
    cleanups = 0;
  }
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

void Server::run() {
  // RME_SERVE_TRACE=1 prints one line per launch to stderr: frames, queue
  // left behind, and the host-side split of the launch's time.
  const bool trace = std::getenv("RME_SERVE_TRACE") && std::getenv("RME_SERVE_TRACE")[0] == '1';
  std::thread copier([this] { copy_loop(); });
  int slot = 0;
  for (;;) {
    Launch L;
    {
      std::unique_lock<std::mutex> lk(m);
      cv.wait(lk, [&] { return stop || !queue.empty() || cleanups > 0; });
      if (cleanups > 0) release_closed();
      if (stop && queue.empty()) break;
      if (queue.empty()) continue;
      // Oldest first, at most kPerStream frames of a stream (in order) and
      // max_frames_per_launch in all.
      std::map<int32_t, int> taken;
      for (auto it = queue.begin(); it != queue.end() && (int)L.batch.size() < o.max_frames_per_launch;) {
        if (taken[it->stream] >= kPerStream) {
          ++it;
          continue;
        }
        ++taken[it->stream];
        L.batch.push_back(std::move(*it));
        it = queue.erase(it);
      }
      L.left = queue.size();
      // The staging buffer of this slot is free once the copier has
      // finished the launch that used it last.
      copied_cv.wait(lk, [&] { return !slot_busy[slot]; });
      slot_busy[slot] = true;
    }
    L.slot = slot;
    L.t_take = now();
    // Upload each frame into its stream's ring of pictures; frames with at
    // least one earlier picture are searched against up to nref of them.
    std::vector<rme_frame> frames;
    std::vector<rme_params> params;
    L.status.assign(L.batch.size(), 0);
    L.count.assign(L.batch.size(), 0);
    L.offset.assign(L.batch.size(), 0);
    std::vector<size_t> searched;
    for (size_t i = 0; i < L.batch.size(); ++i) {
      Stream* st;
      {
        std::lock_guard<std::mutex> lk(m);
        st = &streams[L.batch[i].stream];
      }
      const int slots = st->nref + kPerStream;
      const int32_t pic = st->pic_base + (int32_t)(st->frames % slots);
      int rc = rme_picture_upload(ctx, pic, &st->d, L.batch[i].luma, 1, nullptr);
      if (rc) {
        L.status[i] = rc;
        continue;
      }
      const int nr = (int)std::min<int64_t>(st->nref, st->frames);
      {
        // The worker alone writes `frames`; submits read it under the lock.
        std::lock_guard<std::mutex> lk(m);
        ++st->frames;
      }
      if (nr == 0) continue;
      rme_frame f{};
      f.src_id = pic;
      f.nref = nr;
      for (int r = 0; r < nr; ++r) f.ref_ids[r] = st->pic_base + (int32_t)((st->frames - 2 - r) % slots);
      frames.push_back(f);
      params.push_back(st->p);
      searched.push_back(i);
    }
    L.t_up = now();
    if (!frames.empty()) {
      std::vector<int64_t> offs(frames.size());
      int64_t total = 0;
      for (size_t k = 0; k < frames.size(); ++k) {
        int32_t cnt = 0;
        rme_frame_result_count(ctx, &frames[k], &params[k], &cnt);
        offs[k] = total;
        L.offset[searched[k]] = total;
        L.count[searched[k]] = cnt;
        total += cnt;
      }
      if ((int64_t)staging_n[slot] < total) {
        if (staging[slot]) cudaFreeHost(staging[slot]);
        staging[slot] = nullptr;
        staging_n[slot] = 0;
        if (cudaMallocHost(&staging[slot], sizeof(rme_result) * total) == cudaSuccess) staging_n[slot] = total;
      }
      // Pinned results: the search copies them there directly.
      const int rc = staging[slot] ? rme_batch_search(ctx, frames.data(), params.data(), (int32_t)frames.size(),
                                                      staging[slot], offs.data(), nullptr)
                                   : RME_ENOMEM;
      if (rc)
        for (size_t k = 0; k < frames.size(); ++k) L.status[searched[k]] = rc;
    } else {
      cudaDeviceSynchronize();  // the uploads have read their buffers
    }
    L.t_search = now();
    if (trace)
      std::fprintf(stderr, "serve: %zu frames (%zu searched), %zu queued; upload %.2f ms, search %.2f ms\n",
                   L.batch.size(), frames.size(), L.left, (L.t_up - L.t_take) * 1e3, (L.t_search - L.t_up) * 1e3);
    {
      std::lock_guard<std::mutex> lk(m);
      copies.push_back(std::move(L));
    }
    copy_cv.notify_one();
    slot ^= 1;
  }
  {
    std::lock_guard<std::mutex> lk(m);
    copier_stop = true;
  }
  copy_cv.notify_one();
  copier.join();
}

// The copier thread: results of finished launches into the requests'
// buffers, then their completions, while the worker runs the next launch.
void Server::copy_loop() {
  for (;;) {
    Launch L;
    {
      std::unique_lock<std::mutex> lk(m);
      copy_cv.wait(lk, [&] { return copier_stop || !copies.empty(); });
      if (copies.empty()) return;
      L = std::move(copies.front());
      copies.pop_front();
    }
    for (size_t i = 0; i < L.batch.size(); ++i)
      if (L.status[i] == 0 && L.count[i] > 0)
        std::memcpy(L.batch[i].out, staging[L.slot] + L.offset[i], sizeof(rme_result) * L.count[i]);
    const double t = now();
    std::lock_guard<std::mutex> lk(m);
    for (size_t i = 0; i < L.batch.size(); ++i) {
      rme_completion c{};
      c.request_id = L.batch[i].id;
      c.stream_id = L.batch[i].stream;
      c.status = L.status[i];
      c.submit_s = L.batch[i].submit_s;
      c.done_s = t;
      c.nresults = L.status[i] == 0 ? (int32_t)L.count[i] : 0;
      done.push_back(c);
      pool[L.batch[i].bytes].push_back(L.batch[i].luma);
      Stream& st = streams[L.batch[i].stream];
      if (--st.pending == 0 && st.closing) ++cleanups;
    }
    slot_busy[L.slot] = false;
    copied_cv.notify_all();
    if (cleanups) cv.notify_one();
  }
}

}  // namespace

extern "C" {

int rme_serve_start(void* ctx, const rme_serve_opts* o, void** server) {
  if (!ctx || !o || !server || o->max_frames_per_launch < 1 || o->max_frames_per_launch > 255 || o->max_streams < 1)
    return RME_EINVAL;
  auto* s = new Server();
  s->ctx = ctx;
  s->o = *o;
  s->worker = std::thread([s] { s->run(); });
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
  std::lock_guard<std::mutex> lk(s->m);
  if (s->streams.count(stream_id)) return RME_EINVAL;
  if ((int)s->streams.size() >= s->o.max_streams || s->resident + bytes > s->o.hbm_budget_bytes) return RME_EBUSY;
  Stream st;
  st.d = *d;
  st.p = *p;
  st.nref = nref;
  st.bytes = bytes;
  st.pic_base = s->next_pic_base;
  s->next_pic_base += RME_MAX_REFS + kPerStream;
  s->resident += bytes;
  s->streams[stream_id] = st;
  return RME_OK;
}

int rme_serve_submit(void* server, int32_t stream_id, const void* luma, rme_result* out, int64_t* request_id) {
  auto* s = (Server*)server;
  if (!s || !luma) return RME_EINVAL;
  Request r;
  r.submit_s = s->now();
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->streams.find(stream_id);
  if (it == s->streams.end() || it->second.closing) return RME_ENOTFOUND;
  const rme_picture_desc& d = it->second.d;
  r.bytes = (size_t)d.stride * d.height * (d.bit_depth == 8 ? 1 : 2);
  if ((it->second.frames > 0 || it->second.pending > 0) && !out) return RME_EINVAL;  // this frame is searched
  r.luma = s->take_buffer(r.bytes);
  if (!r.luma) return RME_ENOMEM;
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
    // The worker releases its pictures once its last request completes.
    it->second.closing = true;
    ++s->cleanups;
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
  for (auto& kv : s->streams)
    for (int k = 0; k < kv.second.nref + kPerStream; ++k) rme_picture_release(s->ctx, kv.second.pic_base + k);
  for (auto& q : s->queue) cudaFreeHost(q.luma);
  for (int k = 0; k < 2; ++k)
    if (s->staging[k]) cudaFreeHost(s->staging[k]);
  for (auto& kv : s->pool)
    for (void* b : kv.second) cudaFreeHost(b);
  delete s;
  return RME_OK;
}

}  // extern "C"
