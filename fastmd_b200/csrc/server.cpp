// Continuous-batching request server over one mixed-precision batch.
//
// A pool of generator threads parses each submitted request and builds its
// melt on the host; the batch thread receives them in submission order.  The batch thread owns the batch: each
// round it admits generated requests while replica slots and the
// device-memory budget allow, advances every resident replica by
// steps_per_round steps in the shared CUDA-graph step loop (new replicas run
// their capped push-off in the same steps, beside the others), retires the
// replicas that reached their run.conf nsteps (or faulted), publishes their
// results, and back-fills the freed slots in the next round.  A replica's
// trajectory does not depend on what else is resident (chunk-aligned
// segments, per-replica reductions and rebuild decisions).
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <algorithm>
#include <deque>
#include <map>
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

// A request whose melt has been generated off the batch thread.
struct Prepared {
  Request rq;
  fmd::RunConfig cfg;
  fmd::Topology topo;
  int64_t bytes = 0;
  fmd_status error = FMD_OK;
};

struct Running {
  int64_t id;
  int slot;
  int32_t natoms;
  int64_t target;
  double submit, start;
  int64_t last_step;
  bool pushing;  // capped push-off still running (its steps are not counted)
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
  std::condition_variable cv, gen_cv;
  std::deque<Request> queue;   // submitted, not taken by a generator
  std::deque<Prepared> ready;  // generated, in submission order, waiting for a slot and memory
  std::map<int64_t, Prepared> out_of_order;  // generated ahead of an earlier request
  int64_t next_ready = 1;      // id of the next request to move into ready
  std::vector<Running> running;
  std::deque<fmd_request_result> done;
  std::atomic<bool> stop{false};
  std::thread th;
  std::vector<std::thread> gen_th;
  int64_t next_id = 1;
  int64_t finished = 0;
  double atom_steps = 0;
  double t0 = 0;
  std::string fatal;
  // host seconds per phase of the batch thread, rounds
  double t_admit = 0, t_run = 0, t_retire = 0;
  int64_t rounds = 0;

  void publish_error(const Request& rq, fmd_status code) {
    fmd_request_result res{};
    res.request_id = rq.id;
    res.status = code;
    res.submit_time = rq.submit - t0;
    res.finish_time = now_s() - t0;
    std::lock_guard<std::mutex> lk(mu);
    done.push_back(res);
    ++finished;
  }

  // Melt generation, parsing and sizing on a pool of host threads; results
  // reach the batch thread in submission order, so it only uploads and steps.
  void generate() {
    while (!stop.load()) {
      Request rq;
      {
        std::unique_lock<std::mutex> lk(mu);
        gen_cv.wait_for(lk, std::chrono::milliseconds(20), [&] { return !queue.empty() || stop.load(); });
        if (queue.empty()) continue;
        rq = queue.front();
        queue.pop_front();
      }
      Prepared p;
      p.rq = rq;
      try {
        p.cfg = fmd::parse_run_conf(rq.conf);
        p.topo = fmd::generate_melt(rq.gen);
        fmd::validate(p.cfg, p.topo);
        const auto plan = fmd::mixed::plan_replica(p.cfg, p.topo.natoms, p.topo.box_L);
        p.bytes = fmd::mixed::estimate_bytes(plan, p.topo.nbonds(), p.topo.nangles());
      } catch (const fmd::Error& e) {
        p.error = e.code;
      } catch (const std::exception&) {
        p.error = FMD_ERR_ARG;
      }
      std::lock_guard<std::mutex> lk(mu);
      out_of_order.emplace(p.rq.id, std::move(p));
      for (auto it = out_of_order.find(next_ready); it != out_of_order.end(); it = out_of_order.find(next_ready)) {
        ready.push_back(std::move(it->second));
        out_of_order.erase(it);
        ++next_ready;
      }
      cv.notify_one();
    }
  }

  void loop() {
    cudaSetDevice(device);
    while (!stop.load()) {
      {
        std::unique_lock<std::mutex> lk(mu);
        if (ready.empty() && running.empty()) {
          cv.wait_for(lk, std::chrono::milliseconds(20));
          continue;
        }
      }
      // ---- admission: generated requests, while slots and memory allow
      const double ta = now_s();
      for (;;) {
        Prepared p;
        {
          std::lock_guard<std::mutex> lk(mu);
          if (ready.empty()) break;
          if (ready.front().error == FMD_OK && batch->bytes_in_use() + ready.front().bytes > batch->budget_bytes() &&
              !running.empty())
            break;  // wait for memory
          p = std::move(ready.front());
          ready.pop_front();
        }
        if (p.error != FMD_OK) {
          publish_error(p.rq, p.error);
          continue;
        }
        try {
          const int64_t natoms = p.topo.natoms;
          int slot;
          try {
            slot = batch->add(p.cfg, p.topo, &p.rq.gen);
          } catch (const fmd::Error& e) {
            if (e.code == FMD_ERR_CAPACITY && !running.empty()) {
              // back-fill later, first in line
              std::lock_guard<std::mutex> lk(mu);
              ready.push_front(std::move(p));
              break;
            }
            throw;
          }
          Running r;
          r.id = p.rq.id;
          r.slot = slot;
          r.natoms = (int32_t)natoms;
          r.target = p.cfg.nsteps;
          r.submit = p.rq.submit;
          r.start = now_s();
          r.last_step = 0;
          r.pushing = batch->pushoff_pending(slot) > 0;
          std::lock_guard<std::mutex> lk(mu);
          running.push_back(r);
        } catch (const fmd::Error& e) {
          publish_error(p.rq, e.code);
        } catch (const std::exception&) {
          publish_error(p.rq, FMD_ERR_ARG);
        }
      }
      t_admit += now_s() - ta;
      if (running.empty()) continue;
      // ---- advance every resident replica (push-offs alongside)
      const double tr = now_s();
      try {
        batch->run(steps_per_round, true);
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu);
        fatal = e.what();
        stop = true;
        break;
      }
      t_run += now_s() - tr;
      ++rounds;
      // ---- retire finished / faulted replicas
      const double tt = now_s();
      std::vector<Running> keep;
      for (auto& r : running) {
        const auto& R = batch->rep(r.slot);
        if (r.pushing) {
          if (R.status == 0 && batch->pushoff_pending(r.slot) > 0) {
            keep.push_back(r);
            continue;
          }
          r.pushing = false;  // its run starts at step 0
          r.last_step = 0;
        }
        atom_steps += (double)r.natoms * (double)(R.step - r.last_step);
        r.last_step = R.step;
        const bool fault = R.status != 0;
        if (R.step >= r.target || fault) {          fmd_request_result res{};
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
      t_retire += now_s() - tt;
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
    s->batch->set_concurrent_pushoff(true);
    s->t0 = now_s();
    s->th = std::thread([p = s.get()] { p->loop(); });
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const int ngen = (int)std::min(8u, hw / 2);
    for (int k = 0; k < ngen; ++k) s->gen_th.emplace_back([p = s.get()] { p->generate(); });
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
    s->gen_cv.notify_one();
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
    if (queued) *queued = s->next_id - s->next_ready + (int64_t)s->ready.size();
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

FMD_API fmd_status fmd_server_timing(fmd_server* s, double* admit_s, double* run_s, double* retire_s, int64_t* rounds,
                                     int64_t* graph_captures) {
  return guarded([&] {
    if (!s) throw fmd::Error(FMD_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (admit_s) *admit_s = s->t_admit;
    if (run_s) *run_s = s->t_run;
    if (retire_s) *retire_s = s->t_retire;
    if (rounds) *rounds = s->rounds;
    if (graph_captures) *graph_captures = s->batch->graph_captures();
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
        if (s->queue.empty() && s->ready.empty() && s->out_of_order.empty() && s->running.empty() &&
            s->next_ready == s->next_id)
          return;
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
    s->gen_cv.notify_all();
    if (s->th.joinable()) s->th.join();
    for (auto& t : s->gen_th)
      if (t.joinable()) t.join();
    delete s;
  });
}

// ------------------------------------------------------------ several GPUs
// Greedy longest-processing-time placement: items in decreasing cost (ties:
// lower index first), each to the part with the least total cost so far
// (ties: lower part index).  Deterministic, so every rank of a multi-process
// run computes the same assignment.
FMD_API fmd_status fmd_partition_replicas(const int64_t* cost, int32_t n, int32_t nparts, int32_t* part_of,
                                          int64_t* part_cost) {
  return guarded([&] {
    if (n < 0 || nparts <= 0 || (n > 0 && (!cost || !part_of))) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    std::vector<int32_t> order(n);
    for (int32_t i = 0; i < n; ++i) {
      if (cost[i] < 0) throw fmd::Error(FMD_ERR_ARG, "negative cost");
      order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
    std::vector<int64_t> load(nparts, 0);
    for (int32_t i : order) {
      int32_t best = 0;
      for (int32_t p = 1; p < nparts; ++p)
        if (load[p] < load[best]) best = p;
      part_of[i] = best;
      load[best] += cost[i];
    }
    if (part_cost)
      for (int32_t p = 0; p < nparts; ++p) part_cost[p] = load[p];
  });
}

}  // extern "C"

// A request server per device; requests go to the server with the least
// outstanding work (atoms x steps submitted and not yet polled).
struct fmd_server_pool {
  std::vector<fmd_server*> servers;
  std::vector<int32_t> devices;
  std::vector<int64_t> work;  // outstanding atoms x steps per server
  std::mutex mu;
  int64_t next_id = 1;
  std::map<std::pair<int, int64_t>, std::pair<int64_t, int64_t>> ids;  // (server, local id) -> (pool id, work)
};

extern "C" {

FMD_API fmd_status fmd_server_pool_create(const fmd_server_opts* opts, const int32_t* devices, int32_t ndevices,
                                          fmd_server_pool** out) {
  return guarded([&] {
    if (!out || !devices || ndevices <= 0) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    *out = nullptr;
    std::unique_ptr<fmd_server_pool> p(new fmd_server_pool());
    try {
      for (int32_t k = 0; k < ndevices; ++k) {
        fmd_server_opts o{};
        if (opts) o = *opts;
        o.batch.device = devices[k];
        fmd_server* s = nullptr;
        const fmd_status st = fmd_server_create(&o, &s);
        if (st != FMD_OK) throw fmd::Error(st, "server on device " + std::to_string(devices[k]) + " failed");
        p->servers.push_back(s);
        p->devices.push_back(devices[k]);
        p->work.push_back(0);
      }
    } catch (...) {
      for (fmd_server* s : p->servers) fmd_server_destroy(s);
      throw;
    }
    *out = p.release();
  });
}

FMD_API fmd_status fmd_server_pool_submit(fmd_server_pool* p, const char* conf, const fmd_melt_spec* gen,
                                          int64_t* request_id, int32_t* server) {
  return guarded([&] {
    if (!p || !conf || !gen || !request_id) throw fmd::Error(FMD_ERR_ARG, "null argument");
    const fmd::RunConfig cfg = fmd::parse_run_conf(conf);
    const int64_t w = (int64_t)gen->nchains * gen->chain_length * std::max<int64_t>(1, cfg.nsteps);
    std::lock_guard<std::mutex> lk(p->mu);
    int best = 0;
    for (int k = 1; k < (int)p->servers.size(); ++k)
      if (p->work[k] < p->work[best]) best = k;
    int64_t local = 0;
    const fmd_status st = fmd_server_submit(p->servers[best], conf, gen, &local);
    if (st != FMD_OK) {
      char buf[512] = {0};
      fmd_last_error(buf, sizeof(buf));
      throw fmd::Error(st, buf);
    }
    const int64_t id = p->next_id++;
    p->ids[{best, local}] = {id, w};
    p->work[best] += w;
    *request_id = id;
    if (server) *server = best;
  });
}

FMD_API fmd_status fmd_server_pool_poll(fmd_server_pool* p, fmd_request_result* out, int32_t cap, int32_t* n) {
  return guarded([&] {
    if (!p || !n || (cap > 0 && !out)) throw fmd::Error(FMD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(p->mu);
    int32_t got = 0;
    for (int k = 0; k < (int)p->servers.size() && got < cap; ++k) {
      int32_t m = 0;
      const fmd_status st = fmd_server_poll(p->servers[k], out + got, cap - got, &m);
      if (st != FMD_OK) throw fmd::Error(st, "poll failed");
      for (int32_t q = got; q < got + m; ++q) {
        auto it = p->ids.find({k, out[q].request_id});
        if (it == p->ids.end()) throw fmd::Error(FMD_ERR_STATE, "unknown request in a pooled server");
        out[q].request_id = it->second.first;
        p->work[k] -= it->second.second;
        p->ids.erase(it);
      }
      got += m;
    }
    *n = got;
  });
}

FMD_API fmd_status fmd_server_pool_stats(fmd_server_pool* p, int64_t* queued, int64_t* running, int64_t* finished,
                                         int64_t* atoms_resident, double* atom_steps) {
  return guarded([&] {
    if (!p) throw fmd::Error(FMD_ERR_ARG, "null pool");
    int64_t q = 0, r = 0, f = 0, a = 0;
    double s = 0;
    for (fmd_server* sv : p->servers) {
      int64_t q1 = 0, r1 = 0, f1 = 0, a1 = 0;
      double s1 = 0;
      const fmd_status st = fmd_server_stats(sv, &q1, &r1, &f1, &a1, &s1);
      if (st != FMD_OK) throw fmd::Error(st, "stats failed");
      q += q1;
      r += r1;
      f += f1;
      a += a1;
      s += s1;
    }
    if (queued) *queued = q;
    if (running) *running = r;
    if (finished) *finished = f;
    if (atoms_resident) *atoms_resident = a;
    if (atom_steps) *atom_steps = s;
  });
}

FMD_API fmd_status fmd_server_pool_drain(fmd_server_pool* p, double timeout_s) {
  return guarded([&] {
    if (!p) throw fmd::Error(FMD_ERR_ARG, "null pool");
    const double t_end = now_s() + timeout_s;
    for (fmd_server* sv : p->servers) {
      const fmd_status st = fmd_server_drain(sv, std::max(0.0, t_end - now_s()));
      if (st != FMD_OK) {
        char buf[512] = {0};
        fmd_last_error(buf, sizeof(buf));
        throw fmd::Error(st, buf);
      }
    }
  });
}

FMD_API fmd_status fmd_server_pool_destroy(fmd_server_pool* p) {
  return guarded([&] {
    if (!p) return;
    for (fmd_server* s : p->servers) fmd_server_destroy(s);
    delete p;
  });
}

}  // extern "C"
