// Host-side batch manager for the mixed-precision engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <vector>

#include "dev_common.cuh"
#include "host.h"
#include "mixed.cuh"

namespace fmd {
namespace mixed {

// First-fit segment allocator over [0, capacity) in caller units.
class SegAlloc {
 public:
  void reset(int64_t capacity) {
    free_.clear();
    used_.clear();
    if (capacity > 0) free_[0] = capacity;
    hwm_ = 0;
  }
  int64_t alloc(int64_t n);
  void release(int64_t at);
  int64_t hwm() const { return hwm_; }

 private:
  std::map<int64_t, int64_t> free_, used_;
  int64_t hwm_ = 0;
};

struct ReplicaPlan {
  int G_alloc = 1, P = 1;
  int64_t ncell = 1;
  int32_t slot_cap = 0, nchunks = 0, M = 0;
  int64_t nbr_entries = 0;
};

struct BatchCaps {
  int64_t slots = 0, nbr = 0, cells = 0, bonds = 0, angles = 0;
};

ReplicaPlan plan_replica(const RunConfig& cfg, int32_t natoms, double L);
int64_t estimate_bytes(const ReplicaPlan& p, int32_t nbonds, int32_t nangles);

struct ReplicaInfo {
  bool used = false;
  ReplicaPlan plan;
  RunConfig cfg;
  std::vector<int32_t> type, mol;
  Topology topo;  // bonds, angles, types, masses (positions live on the device)
  int64_t bytes = 0;
  int64_t seg_chunk = -1, seg_cell = -1, seg_nbr = -1, seg_bond = -1, seg_angle = -1;
  int64_t pending_pushoff = 0;
};

class Batch {
 public:
  Batch(const fmd_batch_opts& o, const BatchCaps* exact = nullptr);
  ~Batch();
  int add(const RunConfig& cfg, Topology t, const fmd_melt_spec* pushoff);
  void run(int64_t nsteps, bool respect_nsteps);
  void retire(int r);
  const Rep& rep(int r) const;
  bool used(int r) const { return r >= 0 && r < max_reps_ && info_[r].used; }
  int max_reps() const { return max_reps_; }
  const RunConfig& cfg(int r) const { return info_[r].cfg; }
  void get_state(int r, double* xyz, double* vel, int32_t* image);
  void write_restart(int r, const std::string& path);
  // Restart checkpoint / resume of replica r (see SimEngine::checkpoint).
  void checkpoint(int r, Topology& t, StateFile& s);
  void restore(int r, const Topology& t, const StateFile& s);
  // Server mode: push-offs advance inside run() beside the running replicas
  // instead of freezing them first.
  void set_concurrent_pushoff(bool on) { concurrent_pushoff_ = on; }
  int64_t pushoff_pending(int r) const { return info_[r].pending_pushoff; }
  int64_t graph_captures() const { return graph_captures_; }
  void launch_counts(int64_t* counts, int n);
  void read_state(int r, double* xyz, double* vel, int32_t* image, bool rewrap);
  void force_frame(int r, double* xyz, double* box);
  // Queue a trajectory frame of replica r on the batch stream: positions
  // (id order, wrapped in the last pre-force box) packed into d_xyz, copied
  // to the pinned h_xyz; ready is recorded after the copy.
  void pack_frame(int r, float* d_xyz, float* h_xyz, cudaEvent_t ready);
  // Stress autocorrelation rows (lag in steps, 6 values per row, samples).
  void stress_acf(int r, std::vector<int64_t>& lag, std::vector<double>& val, std::vector<int64_t>& cnt);
  void write_stress_acf(int r, const std::string& path);
  void set_state(int r, const double* xyz, const double* vel, const int32_t* image);
  void forces(int r, double* f, double* pe, double* vir);
  void thermo(int r, fmd_thermo_row* row);
  double rg(int r);
  int64_t pairs(int r, int32_t* pi, int32_t* pj, int64_t cap);
  void totals(int32_t* active, int64_t* atoms, int64_t* bytes);
  void check_status(int r, bool throw_on_fault);
  void ensure_ev(int r);
  // Run the capped-force push-off of every replica admitted with one, batched.
  void finish_pushoffs();
  void complete_pushoffs(const std::vector<int>& pend);
  void complete_done_pushoffs();
  int64_t budget_bytes() const { return budget_bytes_; }
  int64_t bytes_in_use() const { return bytes_in_use_; }
  cudaStream_t stream() const { return st_; }
  Dev dev() const;
  int nchunks_launch() const;
  int nreps_launch() const;
  StepShape shape() const;
  void write_rebuild_list(const std::vector<int>& rs, int rebuilds = -1);  // rebuilds < 0: all listed
  int graph_steps() const { return graph_steps_; }
  void set_max_between(int r, int k);
  void set_list_prune(int r, double delta);
  void set_list_buffer(int r, double skin);
  void mark(int which);
  double elapsed_ms();
  // steady: time the flavour each replica needs on ordinary steps (energies
  // only for NPT), not the one its current step needs (a thermo step).
  double time_force(int iters, int variant = -1, bool steady = false);
  int autotune(int iters, double* ms_out, int cap);
  double time_rebuild(int iters, int variant);
  int nbr_variant() const { return nbr_variant_; }
  const double* nbr_variant_ms() const { return nbr_ms_; }
  int force_variant() const { return force_variant_; }
  // Force / neighbor-list kernel variants for the following steps (< 0: keep).
  void set_variants(int force_variant, int nbr_variant);
  // Forces of the last evaluation as stored (no re-evaluation), id order.
  void last_forces(int r, double* f);
  void list_stats(int64_t* entries, int32_t* max_per_atom);

 private:
  void download_reps();
  void download_reps_keep(int r);
  void upload_reps();
  void freeze_others(int r);
  void upload_atoms(int r, const double* xyz, const double* vel, const int32_t* image);
  void setup(const std::vector<int>& rs);
  void advance_direct(int64_t nsteps);
  void ensure_graph();

  int device_ = 0;
  cudaStream_t st_ = nullptr;
  cudaStream_t side_ = nullptr;    // captures conditional-node bodies
  cudaStream_t side_hi_ = nullptr;  // captures the rebuild branches' bodies (high priority)
  cudaStream_t branch_[4] = {};     // further branches of a captured step
  int graph_steps_ = 50;
  int force_variant_ = 0;
  bool concurrent_pushoff_ = false;
  int hw_nreps_ = 0, hw_cells_ = 0, hw_home_ = 0;  // layout high-water marks
  int slot_cap_chunks_ = 0;                        // chunks the per-chunk arrays hold
  StepShape graph_shape_{};
  int64_t graph_captures_ = 0;
  int nbr_variant_ = 0;
  double nbr_ms_[kNbrVariants] = {0, 0, 0};
  int max_reps_ = 256;
  BatchCaps caps_;
  int64_t budget_bytes_ = 0, bytes_in_use_ = 0, bytes_ = 0;
  SegAlloc slot_alloc_, cell_alloc_, nbr_alloc_, bond_alloc_, angle_alloc_;
  DevBuf<float4> pos_, vel_, force_, ref_, tpos_, tvel_;
  DevBuf<int4> img_, timg_;
  DevBuf<uint32_t> key_;
  DevBuf<int32_t> perm_, bucket_, slot_of_, boff_, aoff_, ncnt_, tcnt_, pcnt_;
  DevBuf<uint32_t> bnd_;
  DevBuf<uint2> ang_;
  DevBuf<double> part_;
  DevBuf<unsigned long long> kcount_;
  DevBuf<double> acf_;  // stress autocorrelator state per replica slot
  DevBuf<float2> tab_;  // pair-table points of every replica (appended at add)
  std::vector<float2> tab_host_;
  DevBuf<int> rb_;  // rebuild work list
  std::vector<int> wl_;  // host staging of a host-written work list (kept alive for the async copy)
  int host_mode_ = 0;  // rebuild form of the current step, read back by direct-launch steps
  DevBuf<int32_t> cell_cnt_, cell_start_, cell_fill_;
  DevBuf<int2> bent_;
  DevBuf<int4> aent_;
  DevBuf<uint32_t> nbr_, pnbr_;  // full (rc + skin) and pruned (rc + prune_delta) lists
  DevBuf<Rep> reps_;
  DevBuf<int4> chunk_rep_;
  std::vector<int4> h_chunk_rep_;
  std::vector<Rep> h_reps_;
  std::vector<ReplicaInfo> info_;
  cudaGraphExec_t graph_exec_ = nullptr;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  bool graph_dirty_ = true;
};

}  // namespace mixed
}  // namespace fmd
