// Engine interface shared by the FP64 plain form and the mixed batched form.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "host.h"
#include "traj.h"

namespace fmd {

class SimEngine {
 public:
  virtual ~SimEngine() = default;
  virtual void step(int64_t nsteps) = 0;
  virtual void compute_forces(double* f, double* pe, double* vir) = 0;
  virtual void get_state(double* xyz, double* vel, int32_t* image) = 0;
  virtual void set_state(const double* xyz, const double* vel, const int32_t* image) = 0;
  virtual void thermo(fmd_thermo_row* row) = 0;
  virtual double rg() = 0;
  virtual int64_t pairs(int32_t* pi, int32_t* pj, int64_t cap) = 0;
  virtual int32_t natoms() const = 0;
  virtual int32_t nbonds() const = 0;
  virtual int32_t nangles() const = 0;
  virtual int64_t step_count() const = 0;
  virtual double box_L() = 0;
  virtual int64_t rebuilds() const = 0;
  virtual int32_t status_word() = 0;
  virtual int32_t max_neighbors() const = 0;
  // Stress autocorrelation rows (run.conf 'stress'); the mixed form keeps the
  // correlator on the device.
  virtual void stress_acf(std::vector<int64_t>& lag, std::vector<double>& val, std::vector<int64_t>& cnt) {
    (void)lag;
    (void)val;
    (void)cnt;
    throw Error(FMD_ERR_ARG, "the stress autocorrelation is computed by the mixed form");
  }
  // One trajectory frame of the current state (positions wrapped in the box
  // of the last pre-force update, the current box edge).
  virtual void dump_frame(TrajWriter& w) {
    std::vector<double> x(3 * (size_t)natoms());
    get_state(x.data(), nullptr, nullptr);
    w.write_host(step_count(), box_L(), x.data());
  }
  // Restart checkpoint: fills t's positions, velocities, image flags and box
  // (data-file order) and the sidecar values; the engine then continues from
  // exactly the state restore() gives a resumed run (positions re-loaded from
  // those FP64 values, list rebuilt, forces re-evaluated), so the run after a
  // checkpoint is the same whether the process continues or resumes.
  virtual void checkpoint(Topology& t, StateFile& s) = 0;
  // Resume: the state of a data file (t) and its sidecar.
  virtual void restore(const Topology& t, const StateFile& s) = 0;
  virtual void write_stress_acf(const std::string& path) {
    (void)path;
    throw Error(FMD_ERR_ARG, "the stress autocorrelation is computed by the mixed form");
  }
};

// FP64 mirror of the reference step loop (one system, host-driven rebuild test).
std::unique_ptr<SimEngine> make_plain_engine(const RunConfig& cfg, Topology topo, const fmd_melt_spec* pushoff);
// Mixed-precision engine over a one-replica batch.
std::unique_ptr<SimEngine> make_mixed_engine(const RunConfig& cfg, Topology topo, const fmd_melt_spec* pushoff);

}  // namespace fmd
