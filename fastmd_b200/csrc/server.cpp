// Continuous-batching request server over one mixed-precision batch.
//
// A host thread owns the batch.  Each round it admits queued requests while
// replica slots and the device-memory budget allow (generation and optional
// push-off happen at admission), advances every resident replica by
// steps_per_round steps in the shared CUDA-graph step loop, retires the
// replicas that reached their run.conf nsteps (or faulted), publishes their
// results, and back-fills the freed slots in the next round.  A replica's
// trajectory does not depend on what else is resident (chunk-aligned
// segments, per-replica reductions and rebuild decisions).
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch.h"
#include "host.h"

namespace {

struct Request {
  int64_t id;
  std::string conf;
  fmd_melt_spec gen;
  double submit;
};

struct Running {
  int64_t id;
  int slot;
  int32_t natoms;
  int64_t target;
  double submit, start;
  int64_t last_step;
};

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct fmd_server {
  std::unique_ptr<fmd::mixed::Batch> batch;
  int32_t steps_per_round = 200;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request> queue;
  std::vector<Running> running;
  std::deque<fmd_request_result> done;
  std::atomic<bool> stop{false};
  std::thread th;
  int64_t next_id = 1;
  int64_t finished = 0;
  double atom_steps = 0;
  double t0 = 0;
  std::string fatal;

  void loop() {
    cudaSetDevice(device);
    while (!stop.load()) {
      // ---- admission
      std::vector<Request> admit;
      {
        std::unique_lock<std::mutex> lk(mu);
        if (queue.empty() && running.empty()) {
          cv.wait_for(lk, std::chrono::milliseconds(20));
          continue;
        }
      }
      for (;;) {
        Request rq;
        {
          std::lock_guard<std::mutex> lk(mu);
          if (queue.empty()) break;
          rq = queue.front();
        }
        fmd_request_result res{};
        res.request_id = rq.id;
        res.submit_time = rq.submit - t0;
        try {
          fmd::RunConfig cfg = fmd::parse_run_conf(rq.conf);
          const int64_t n = (int64_t)rq.gen.nchains * rq.gen.chain_length;
          const double L = std::cbrt((double)n / rq.gen.density);
          const auto plan = fmd::mixed::plan_replica(cfg, (int32_t)n, L);
          const int64_t need = fmd::mixed::estimate_bytes(plan, (int32_t)n, (int32_t)n);
          if (batch->bytes_in_use() + need > batch->budget_bytes() && !running.empty()) break;  // wait for memory
          fmd::Topology t = fmd::generate_melt(rq.gen);
          fmd::validate(cfg, t);
          int slot;
          try {
            slot = batch->add(cfg, std::move(t), &rq.gen);
          } catch (const fmd::Error& e) {
            if (e.code == FMD_ERR_CAPACITY && !running.empty()) break;  // back-fill later
            throw;
          }
          Running r;
          r.id = rq.id;
          r.slot = slot;
          r.natoms = (int32_t)n;
          r.target = cfg.nsteps;
          r.submit = rq.submit;
          r.start = now_s();
          r.last_step = 0;
          std::lock_guard<std::mutex> lk(mu);
          queue.pop_front();
          running.push_back(r);
        } catch (const fmd::Error& e) {
          res.status = e.code;
          res.finish_time = now_s() - t0;
          std::lock_guard<std::mutex> lk(mu);
          queue.pop_front();
          done.push_back(res);
          ++finished;
        } catch (const std::exception& e) {
          res.status = FMD_ERR_ARG;
          res.finish_time = now_s() - t0;
          std::lock_guard<std::mutex> lk(mu);
          queue.pop_front();
          done.push_back(res);
          ++finished;
        }
      }
      if (running.empty()) continue;
      // ---- advance every resident replica
      try {
        batch->run(steps_per_round, true);
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu);
        fatal = e.what();
        stop = true;
        break;
      }
      // ---- retire finished / faulted replicas
      std::vector<Running> keep;
      for (auto& r : running) {
        const auto& R = batch->rep(r.slot);
        atom_steps += (double)r.natoms * (double)(R.step - r.last_step);
        r.last_step = R.step;
        const bool fault = R.status != 0;
        if (R.step >= r.target || fault) {
          fmd_request_result res{};
          res.request_id = r.id;
          res.status = fault ? FMD_ERR_FAULT : FMD_OK;
          res.natoms = r.natoms;
          res.steps = R.step;
          res.submit_time = r.submit - t0;
          res.start_time = r.start - t0;
          try {
            batch->thermo(r.slot, &res.thermo);
            res.rg = batch->rg(r.slot);
            batch->retire(r.slot);
          } catch (const std::exception&) {
            res.status = FMD_ERR_CUDA;
          }
          res.finish_time = now_s() - t0;
          std::lock_guard<std::mutex> lk(mu);
          done.push_back(res);
          ++finished;
        } else {
          keep.push_back(r);
        }
      }
      std::lock_guard<std::mutex> lk(mu);
      running.swap(keep);
    }
  }
};

namespace {
template <typename F>
fmd_status guarded(F&& f) {
  try {
    f();
    fmd::set_last_error("");
    return FMD_OK;
  } catch (const fmd::Error& e) {
    fmd::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    fmd::set_last_error(e.what());
    return FMD_ERR_ARG;
  }
}
}  // namespace

extern "C" {

FMD_API fmd_status fmd_server_create(const fmd_server_opts* opts, fmd_server** out) {
  return guarded([&] {
    if (!out) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      throw fmd::Error(FMD_ERR_NO_DEVICE, "no CUDA device available");
    }
    fmd_server_opts o{};
    if (opts) o = *opts;
    std::unique_ptr<fmd_server> s(new fmd_server());
    s->device = o.batch.device;
    s->steps_per_round = o.steps_per_round > 0 ? o.steps_per_round : 200;
    s->batch.reset(new fmd::mixed::Batch(o.batch));
    s->t0 = now_s();
    s->th = std::thread([p = s.get()] { p->loop(); });
    *out = s.release();
  });
}

FMD_API fmd_status fmd_server_submit(fmd_server* s, const char* conf, const fmd_melt_spec* gen, int64_t* request_id) {
  return guarded([&] {
    if (!s || !conf || !gen || !request_id) throw fmd::Error(FMD_ERR_ARG, "null argument");
    fmd::parse_run_conf(conf);  // reject bad text at submission
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->fatal.empty()) throw fmd::Error(FMD_ERR_STATE, "server stopped: " + s->fatal);
    Request r{s->next_id++, conf, *gen, now_s()};
    s->queue.push_back(r);
    *request_id = r.id;
    s->cv.notify_one();
  });
}

FMD_API fmd_status fmd_server_poll(fmd_server* s, fmd_request_result* out, int32_t cap, int32_t* n) {
  return guarded([&] {
    if (!s || !n || (cap > 0 && !out)) throw fmd::Error(FMD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    int32_t k = 0;
    while (k < cap && !s->done.empty()) {
      out[k++] = s->done.front();
      s->done.pop_front();
    }
    *n = k;
  });
}

FMD_API fmd_status fmd_server_stats(fmd_server* s, int64_t* queued, int64_t* running, int64_t* finished,
                                    int64_t* atoms_resident, double* atom_steps) {
  return guarded([&] {
    if (!s) throw fmd::Error(FMD_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int64_t)s->queue.size();
    if (running) *running = (int64_t)s->running.size();
    if (finished) *finished = s->finished;
    if (atoms_resident) {
      int64_t a = 0;
      for (auto& r : s->running) a += r.natoms;
      *atoms_resident = a;
    }
    if (atom_steps) *atom_steps = s->atom_steps;
  });
}

FMD_API fmd_status fmd_server_drain(fmd_server* s, double timeout_s) {
  return guarded([&] {
    if (!s) throw fmd::Error(FMD_ERR_ARG, "null server");
    const double t_end = now_s() + timeout_s;
    for (;;) {
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->fatal.empty()) throw fmd::Error(FMD_ERR_STATE, "server stopped: " + s->fatal);
        if (s->queue.empty() && s->running.empty()) return;
      }
      if (now_s() > t_end) throw fmd::Error(FMD_ERR_TIMEOUT, "drain timed out");
      std::this_thread::sleep_for(std::chrono::milliseconds(5));
    }
  });
}

FMD_API fmd_status fmd_server_destroy(fmd_server* s) {
  return guarded([&] {
    if (!s) return;
    s->stop = true;
    s->cv.notify_all();
    if (s->th.joinable()) s->th.join();
    delete s;
  });
}

}  // extern "C"
