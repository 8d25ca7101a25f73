// Binary trajectory writer (the reference's dump format, io/dump.cu:12-56):
// header {int32 magic 0x4D444247, int32 natoms, int32 ntypes}, then per frame
// {int64 step, int32 n, float box_L, float xyz[3 n]}.  Frames are packed on
// the device into one of two pinned buffers and written by a background
// thread, so a dump returns as soon as the copy is queued.
#pragma once
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>

#include <cuda_runtime.h>

#include "host.h"

namespace fmd {
namespace mixed {
class Batch;
}

class TrajWriter {
 public:
  TrajWriter(const std::string& path, int32_t natoms, int32_t ntypes);
  ~TrajWriter();
  // Frame of a batch replica's current state (asynchronous).
  void write(mixed::Batch& b, int r);
  // Frame from host positions (3 n doubles, already wrapped), synchronous copy.
  void write_host(int64_t step, double box_L, const double* xyz);
  // Waits for the queued frames and closes the file; throws on a write error.
  void close();
  int32_t natoms() const { return natoms_; }

 private:
  struct Job {
    int buf;
    int64_t step;
    float L;
    cudaEvent_t ready;  // nullptr: host buffer already filled
  };
  int acquire();  // a free pinned buffer (waits for the writer)
  void loop();

  FILE* f_ = nullptr;
  int32_t natoms_ = 0;
  float* host_[2] = {nullptr, nullptr};
  float* dbuf_ = nullptr;  // device staging of one frame (allocated at the first device frame)
  size_t dbuf_n_ = 0;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  bool busy_[2] = {false, false};
  std::deque<Job> q_;
  std::mutex m_;
  std::condition_variable cv_;
  bool stop_ = false, failed_ = false;
  std::thread th_;
};

}  // namespace fmd

// The C-ABI handle (include/fastmd.h).
struct fmd_traj {
  std::unique_ptr<fmd::TrajWriter> w;
};
