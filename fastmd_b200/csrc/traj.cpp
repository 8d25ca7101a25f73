// Binary trajectory writer (io/dump.cu:12-56 format; see traj.h).
#include "traj.h"

#include <cstring>

#include "batch.h"

namespace fmd {

namespace {
constexpr int32_t kTrajMagic = 0x4D444247;  // dump.cu:25
}

TrajWriter::TrajWriter(const std::string& path, int32_t natoms, int32_t ntypes) : natoms_(natoms) {
  if (natoms <= 0) throw Error(FMD_ERR_ARG, "natoms must be positive");
  f_ = std::fopen(path.c_str(), "wb");
  if (!f_) throw Error(FMD_ERR_IO, "cannot open " + path);
  const int32_t head[3] = {kTrajMagic, natoms, ntypes};
  if (std::fwrite(head, sizeof(int32_t), 3, f_) != 3) {
    std::fclose(f_);
    f_ = nullptr;
    throw Error(FMD_ERR_IO, "cannot write " + path);
  }
  for (int k = 0; k < 2; ++k) {
    FMD_CUDA(cudaHostAlloc(&host_[k], (size_t)natoms * 3 * sizeof(float), cudaHostAllocDefault));
    FMD_CUDA(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming));
  }
  th_ = std::thread([this] { loop(); });
}

TrajWriter::~TrajWriter() {
  try {
    close();
  } catch (...) {
  }
  for (int k = 0; k < 2; ++k) {
    if (host_[k]) cudaFreeHost(host_[k]);
    if (ev_[k]) cudaEventDestroy(ev_[k]);
  }
  if (dbuf_) cudaFree(dbuf_);
}

int TrajWriter::acquire() {
  std::unique_lock<std::mutex> lk(m_);
  cv_.wait(lk, [&] { return !busy_[0] || !busy_[1] || failed_; });
  if (failed_) throw Error(FMD_ERR_IO, "trajectory write failed");
  const int k = busy_[0] ? 1 : 0;
  busy_[k] = true;
  return k;
}

void TrajWriter::write(mixed::Batch& b, int r) {
  if (!f_) throw Error(FMD_ERR_ARG, "trajectory is closed");
  const mixed::Rep& R = b.rep(r);
  if (R.natoms != natoms_) throw Error(FMD_ERR_ARG, "replica size differs from the trajectory's natoms");
  if (!dbuf_) {
    FMD_CUDA(cudaMalloc(&dbuf_, (size_t)natoms_ * 3 * sizeof(float)));
    dbuf_n_ = (size_t)natoms_ * 3;
  }
  const int k = acquire();
  b.pack_frame(r, dbuf_, host_[k], ev_[k]);
  std::lock_guard<std::mutex> lk(m_);
  q_.push_back(Job{k, R.step, (float)R.L, ev_[k]});
  cv_.notify_all();
}

void TrajWriter::write_host(int64_t step, double box_L, const double* xyz) {
  if (!f_) throw Error(FMD_ERR_ARG, "trajectory is closed");
  const int k = acquire();
  for (size_t i = 0; i < (size_t)natoms_ * 3; ++i) host_[k][i] = (float)xyz[i];
  std::lock_guard<std::mutex> lk(m_);
  q_.push_back(Job{k, step, (float)box_L, nullptr});
  cv_.notify_all();
}

void TrajWriter::loop() {
  for (;;) {
    Job j;
    {
      std::unique_lock<std::mutex> lk(m_);
      cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
      if (q_.empty()) return;  // stop requested and nothing left
      j = q_.front();
      q_.pop_front();
    }
    bool ok = true;
    if (j.ready && cudaEventSynchronize(j.ready) != cudaSuccess) ok = false;
    if (ok) {
      const int32_t n = natoms_;
      ok = std::fwrite(&j.step, sizeof(int64_t), 1, f_) == 1 && std::fwrite(&n, sizeof(int32_t), 1, f_) == 1 &&
           std::fwrite(&j.L, sizeof(float), 1, f_) == 1 &&
           std::fwrite(host_[j.buf], sizeof(float), (size_t)n * 3, f_) == (size_t)n * 3;
    }
    std::lock_guard<std::mutex> lk(m_);
    busy_[j.buf] = false;
    if (!ok) failed_ = true;
    cv_.notify_all();
  }
}

void TrajWriter::close() {
  if (!f_) return;
  {
    std::lock_guard<std::mutex> lk(m_);
    stop_ = true;
    cv_.notify_all();
  }
  if (th_.joinable()) th_.join();
  const bool bad = std::fclose(f_) != 0 || failed_;
  f_ = nullptr;
  if (bad) throw Error(FMD_ERR_IO, "trajectory write failed");
}

}  // namespace fmd
