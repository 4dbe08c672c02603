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
// are uploaded. A stream contributes at most one frame per launch; its next
// frame joins the following launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
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
  int32_t pic_base = 0;    // picture ids pic_base .. pic_base + nref
};

struct Request {
  int64_t id = 0;
  int32_t stream = 0;
  std::vector<uint8_t> luma;
  rme_result* out = nullptr;
  double submit_s = 0.0;
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
  std::vector<rme_result> staging;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
  // Release the pictures of closed streams with nothing queued or in flight
  // (worker thread, lock held: only the worker touches the context).
  void release_closed() {
    for (auto it = streams.begin(); it != streams.end();) {
      if (it->second.closing && it->second.pending == 0) {
        for (int k = 0; k <= it->second.nref; ++k) rme_picture_release(ctx, it->second.pic_base + k);
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
  std::vector<Request> batch;
  std::vector<rme_frame> frames;
  std::vector<rme_params> params;
  std::vector<int64_t> offsets, counts;
  std::vector<size_t> searched;  // batch index of each searched frame
  for (;;) {
    batch.clear();
    {
      std::unique_lock<std::mutex> lk(m);
      cv.wait(lk, [&] { return stop || !queue.empty() || cleanups > 0; });
      if (cleanups > 0) release_closed();
      if (stop && queue.empty()) return;
      if (queue.empty()) continue;
      // Oldest first, one frame per stream, at most max_frames_per_launch.
      std::vector<int32_t> taken;
      for (auto it = queue.begin(); it != queue.end() && (int)batch.size() < o.max_frames_per_launch;) {
        if (std::find(taken.begin(), taken.end(), it->stream) != taken.end()) {
          ++it;
          continue;
        }
        taken.push_back(it->stream);
        batch.push_back(std::move(*it));
        it = queue.erase(it);
      }
    }
    // Upload each frame into its stream's ring of pictures; frames with at
    // least one earlier picture are searched against up to nref of them.
    frames.clear();
    params.clear();
    searched.clear();
    std::vector<int> status(batch.size(), 0);
    for (size_t i = 0; i < batch.size(); ++i) {
      Stream* st;
      {
        std::lock_guard<std::mutex> lk(m);
        st = &streams[batch[i].stream];
      }
      const int slots = st->nref + 1;
      const int32_t pic = st->pic_base + (int32_t)(st->frames % slots);
      int rc = rme_picture_upload(ctx, pic, &st->d, batch[i].luma.data(), 1, nullptr);
      if (rc) {
        status[i] = rc;
        continue;
      }
      const int nr = (int)std::min<int64_t>(st->nref, st->frames);
      ++st->frames;
      if (nr == 0) continue;
      rme_frame f{};
      f.src_id = pic;
      f.nref = nr;
      for (int r = 0; r < nr; ++r) f.ref_ids[r] = st->pic_base + (int32_t)((st->frames - 2 - r) % slots);
      frames.push_back(f);
      params.push_back(st->p);
      searched.push_back(i);
    }
    if (!frames.empty()) {
      offsets.assign(frames.size(), 0);
      counts.assign(frames.size(), 0);
      int64_t total = 0;
      for (size_t k = 0; k < frames.size(); ++k) {
        int32_t cnt = 0;
        rme_frame_result_count(ctx, &frames[k], &params[k], &cnt);
        offsets[k] = total;
        counts[k] = cnt;
        total += cnt;
      }
      staging.resize((size_t)std::max<int64_t>(total, 1));
      const int rc = rme_batch_search(ctx, frames.data(), params.data(), (int32_t)frames.size(), staging.data(),
                                      offsets.data(), nullptr);
      for (size_t k = 0; k < frames.size(); ++k) {
        const size_t i = searched[k];
        if (rc) status[i] = rc;
        else std::memcpy(batch[i].out, staging.data() + offsets[k], sizeof(rme_result) * counts[k]);
      }
    }
    const double t = now();
    std::lock_guard<std::mutex> lk(m);
    for (size_t i = 0; i < batch.size(); ++i) {
      rme_completion c{};
      c.request_id = batch[i].id;
      c.stream_id = batch[i].stream;
      c.status = status[i];
      c.submit_s = batch[i].submit_s;
      c.done_s = t;
      c.nresults = 0;
      for (size_t k = 0; k < searched.size(); ++k)
        if (searched[k] == i && status[i] == 0) c.nresults = (int32_t)counts[k];
      done.push_back(c);
      --streams[batch[i].stream].pending;
    }
    release_closed();
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
  const uint64_t bytes = picture_bytes(*d) * (uint64_t)(nref + 1);
  std::lock_guard<std::mutex> lk(s->m);
  if (s->streams.count(stream_id)) return RME_EINVAL;
  if ((int)s->streams.size() >= s->o.max_streams || s->resident + bytes > s->o.hbm_budget_bytes) return RME_EBUSY;
  Stream st;
  st.d = *d;
  st.p = *p;
  st.nref = nref;
  st.bytes = bytes;
  st.pic_base = s->next_pic_base;
  s->next_pic_base += RME_MAX_REFS + 1;
  s->resident += bytes;
  s->streams[stream_id] = st;
  return RME_OK;
}

int rme_serve_submit(void* server, int32_t stream_id, const void* luma, rme_result* out, int64_t* request_id) {
  auto* s = (Server*)server;
  if (!s || !luma) return RME_EINVAL;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->streams.find(stream_id);
  if (it == s->streams.end() || it->second.closing) return RME_ENOTFOUND;
  const rme_picture_desc& d = it->second.d;
  const size_t bytes = (size_t)d.stride * d.height * (d.bit_depth == 8 ? 1 : 2);
  if (it->second.frames > 0 || it->second.pending > 0) {
    if (!out) return RME_EINVAL;  // this frame will be searched
  }
  Request r;
  r.id = ++s->next_id;
  r.stream = stream_id;
  r.luma.assign((const uint8_t*)luma, (const uint8_t*)luma + bytes);
  r.out = out;
  r.submit_s = s->now();
  ++it->second.pending;
  if (request_id) *request_id = r.id;
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
    for (int k = 0; k <= kv.second.nref; ++k) rme_picture_release(s->ctx, kv.second.pic_base + k);
  delete s;
  return RME_OK;
}

}  // extern "C"
