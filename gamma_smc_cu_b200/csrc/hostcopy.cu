// Pinned-ring device -> host copier (see hostcopy.h).
#include "hostcopy.h"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace gsmc {
namespace {

constexpr size_t kSlotBytes = size_t(64) << 20;  // one pinned buffer
constexpr int kSlots = 8;                         // pinned buffers in flight
constexpr size_t kMinPartBytes = size_t(1) << 20;

// FIFO pool of host threads.
class Pool {
 public:
  explicit Pool(int n) {
    for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> l(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void submit(std::function<void()> job) {
    {
      std::lock_guard<std::mutex> l(mu_);
      q_.push_back(std::move(job));
    }
    cv_.notify_one();
  }
  int size() const { return (int)workers_.size(); }

 private:
  void loop() {
    for (;;) {
      std::function<void()> job;
      {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return stop_ || !q_.empty(); });
        if (stop_ && q_.empty()) return;
        job = std::move(q_.front());
        q_.pop_front();
      }
      job();
    }
  }
  std::vector<std::thread> workers_;
  std::deque<std::function<void()>> q_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
};

}  // namespace

struct HostCopier::Impl {
  int device = 0;
  int init_error = cudaSuccess;
  cudaStream_t stream = nullptr;
  struct Slot {
    void* buf = nullptr;
    cudaEvent_t ev = nullptr;
    int pending = 0;  // host jobs still reading buf
  };
  Slot slots[kSlots];
  int next = 0;
  std::mutex mu;  // guards next, pending, error, direct
  std::condition_variable cv;
  int error = cudaSuccess;
  bool direct = false;  // a row too wide for a slot went straight to dst
  std::unique_ptr<Pool> pool;

  void finish_part(Slot& s, int err) {
    std::lock_guard<std::mutex> l(mu);
    if (err != cudaSuccess && error == cudaSuccess) error = err;
    if (--s.pending == 0) cv.notify_all();
  }
};

HostCopier::HostCopier() : impl_(new Impl) {
  Impl& m = *impl_;
  cudaGetDevice(&m.device);
  cudaError_t e = cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking);
  for (int i = 0; i < kSlots && e == cudaSuccess; ++i) {
    e = cudaHostAlloc(&m.slots[i].buf, kSlotBytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m.slots[i].ev, cudaEventDisableTiming);
  }
  m.init_error = e;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  m.pool.reset(new Pool((int)std::min(16u, hw)));
}

HostCopier::~HostCopier() {
  drain();
  Impl& m = *impl_;
  m.pool.reset();
  for (auto& s : m.slots) {
    if (s.ev) cudaEventDestroy(s.ev);
    if (s.buf) cudaFreeHost(s.buf);
  }
  if (m.stream) cudaStreamDestroy(m.stream);
  delete impl_;
}

HostCopier* HostCopier::for_current_device() {
  static std::mutex mu;
  static std::map<int, HostCopier*> copiers;  // live for the process
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> l(mu);
  HostCopier*& c = copiers[dev];
  if (!c) c = new HostCopier();
  return c;
}

int HostCopier::enqueue(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                        size_t rows, cudaEvent_t ready) {
  Impl& m = *impl_;
  if (m.init_error != cudaSuccess) return m.init_error;
  if (rows == 0 || width == 0) return cudaSuccess;
  cudaError_t e = cudaStreamWaitEvent(m.stream, ready, 0);
  if (e != cudaSuccess) return e;
  // A page-locked destination (cudaHostAlloc, cudaHostRegister, the result
  // buffers of gsmc_host_alloc) takes the DMA directly: no staging, no host
  // thread touches the data.
  cudaPointerAttributes attr;
  const bool pinned = cudaPointerGetAttributes(&attr, dst) == cudaSuccess &&
                      attr.type == cudaMemoryTypeHost;
  if (!pinned) cudaGetLastError();  // pageable memory may report an error on older drivers
  if (pinned || width > kSlotBytes) {  // direct: page-locked, or too wide to stage
    {
      std::lock_guard<std::mutex> l(m.mu);
      m.direct = true;
    }
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToHost,
                             m.stream);
  }
  const size_t per = std::max<size_t>(1, kSlotBytes / width);
  for (size_t r0 = 0; r0 < rows; r0 += per) {
    const size_t nr = std::min(per, rows - r0);
    const size_t total = nr * width;
    const bool contiguous = dpitch == width;
    int parts = (int)std::max<size_t>(1, std::min<size_t>(m.pool->size(), total / kMinPartBytes));
    if (!contiguous) parts = (int)std::min<size_t>(parts, nr);
    Impl::Slot* sl;
    {
      // take the next slot once its previous host copy is done, and claim it
      // before releasing the lock
      std::unique_lock<std::mutex> l(m.mu);
      sl = &m.slots[m.next];
      m.next = (m.next + 1) % kSlots;
      m.cv.wait(l, [&] { return sl->pending == 0; });
      sl->pending = parts;
    }
    e = cudaMemcpy2DAsync(sl->buf, width, static_cast<const char*>(src) + r0 * spitch, spitch,
                          width, nr, cudaMemcpyDeviceToHost, m.stream);
    if (e == cudaSuccess) e = cudaEventRecord(sl->ev, m.stream);
    if (e != cudaSuccess) {
      std::lock_guard<std::mutex> l(m.mu);
      sl->pending = 0;
      m.cv.notify_all();
      return e;
    }
    char* d = static_cast<char*>(dst) + r0 * dpitch;
    const char* s = static_cast<const char*>(sl->buf);
    const int dev = m.device;
    for (int p = 0; p < parts; ++p) {
      m.pool->submit([&m, sl, d, s, total, nr, width, dpitch, contiguous, parts, p, dev] {
        cudaSetDevice(dev);
        const int err = cudaEventSynchronize(sl->ev);
        if (err == cudaSuccess) {
          if (contiguous) {
            const size_t a = total * p / parts, b = total * (p + 1) / parts;
            std::memcpy(d + a, s + a, b - a);
          } else {
            const size_t a = nr * p / parts, b = nr * (p + 1) / parts;
            for (size_t r = a; r < b; ++r) std::memcpy(d + r * dpitch, s + r * width, width);
          }
        }
        m.finish_part(*sl, err);
      });
    }
  }
  return cudaSuccess;
}

int HostCopier::record_reads_done(cudaEvent_t ev) {
  Impl& m = *impl_;
  if (m.init_error != cudaSuccess) return m.init_error;
  return cudaEventRecord(ev, m.stream);
}

int HostCopier::drain() {
  Impl& m = *impl_;
  if (m.init_error != cudaSuccess) return m.init_error;
  bool direct;
  {
    std::unique_lock<std::mutex> l(m.mu);
    m.cv.wait(l, [&] {
      for (auto& s : m.slots)
        if (s.pending) return false;
      return true;
    });
    direct = m.direct;
    m.direct = false;
  }
  int err = direct ? cudaStreamSynchronize(m.stream) : cudaSuccess;
  std::lock_guard<std::mutex> l(m.mu);
  if (m.error != cudaSuccess) err = m.error;
  m.error = cudaSuccess;
  return err;
}

}  // namespace gsmc
