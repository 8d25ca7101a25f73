// extern "C" entry points for batches of replicas (include/fastmd.h).
#include <cstring>
#include <memory>
#include <string>

#include "batch.h"
#include "host.h"
#include "traj.h"

struct fmd_batch {
  std::unique_ptr<fmd::mixed::Batch> b;
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
  } catch (const std::bad_alloc&) {
    fmd::set_last_error("host out of memory");
    return FMD_ERR_CAPACITY;
  } catch (const std::exception& e) {
    fmd::set_last_error(e.what());
    return FMD_ERR_ARG;
  }
}

fmd::mixed::Batch& B(fmd_batch* b) {
  if (!b || !b->b) throw fmd::Error(FMD_ERR_ARG, "null batch handle");
  return *b->b;
}

void need_slot(fmd::mixed::Batch& b, int32_t slot) {
  if (!b.used(slot)) throw fmd::Error(FMD_ERR_ARG, "no replica in this slot");
}
}  // namespace

extern "C" {

FMD_API fmd_status fmd_batch_create(const fmd_batch_opts* opts, fmd_batch** out) {
  return guarded([&] {
    if (!out) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      throw fmd::Error(FMD_ERR_NO_DEVICE, "no CUDA device available");
    }
    fmd_batch_opts o{};
    if (opts) o = *opts;
    std::unique_ptr<fmd_batch> b(new fmd_batch());
    b->b.reset(new fmd::mixed::Batch(o));
    *out = b.release();
  });
}

FMD_API fmd_status fmd_batch_destroy(fmd_batch* b) {
  return guarded([&] { delete b; });
}

FMD_API fmd_status fmd_batch_add_replica(fmd_batch* b, const char* conf, const char* data_path,
                                         const fmd_system_desc* desc, const fmd_melt_spec* gen, int32_t* slot) {
  return guarded([&] {
    if (!conf || !slot) throw fmd::Error(FMD_ERR_ARG, "null argument");
    fmd::RunConfig cfg = fmd::parse_run_conf(conf);
    fmd::Topology t = fmd::load_atoms(cfg, data_path, desc, gen);
    // a data file written by fmd_batch_write_restart carries a state sidecar: resume from it
    const std::string data = data_path ? std::string(data_path) : (desc || gen ? std::string() : cfg.data_file);
    fmd::StateFile st;
    const bool resume = !data.empty() && fmd::read_state_file(fmd::state_path(data), st);
    fmd::Topology saved;
    if (resume) saved = t;
    *slot = B(b).add(cfg, std::move(t), gen);
    if (resume) B(b).restore(*slot, saved, st);
  });
}

FMD_API fmd_status fmd_batch_estimate_bytes(const char* conf, int32_t natoms, double box_L, int64_t* bytes) {
  return guarded([&] {
    if (!conf || !bytes || natoms <= 0 || box_L <= 0) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    fmd::RunConfig cfg = fmd::parse_run_conf(conf);
    const auto p = fmd::mixed::plan_replica(cfg, natoms, box_L);
    *bytes = fmd::mixed::estimate_bytes(p, natoms, natoms);
  });
}

FMD_API fmd_status fmd_batch_run(fmd_batch* b, int64_t nsteps) {
  return guarded([&] {
    if (nsteps < 0) throw fmd::Error(FMD_ERR_ARG, "nsteps < 0");
    B(b).run(nsteps, true);
  });
}

FMD_API fmd_status fmd_batch_retire(fmd_batch* b, int32_t slot) {
  return guarded([&] { B(b).retire(slot); });
}

FMD_API fmd_status fmd_batch_replica_info(fmd_batch* b, int32_t slot, fmd_replica_info* info) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!info) throw fmd::Error(FMD_ERR_ARG, "null info");
    const auto& R = bb.rep(slot);
    info->slot = slot;
    info->natoms = R.natoms;
    info->step = R.step;
    info->nsteps = R.nsteps;
    info->status_word = R.status;
    info->active = R.active;
    info->box_L = R.L;
    info->rebuilds = R.rebuilds;
  });
}

FMD_API fmd_status fmd_batch_get_state(fmd_batch* b, int32_t slot, double* xyz, double* vel, int32_t* image) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    bb.get_state(slot, xyz, vel, image);
  });
}

FMD_API fmd_status fmd_batch_write_restart(fmd_batch* b, int32_t slot, const char* path) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!path) throw fmd::Error(FMD_ERR_ARG, "null path");
    bb.write_restart(slot, path);
  });
}

FMD_API fmd_status fmd_batch_thermo(fmd_batch* b, int32_t slot, fmd_thermo_row* row) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!row) throw fmd::Error(FMD_ERR_ARG, "null row");
    bb.thermo(slot, row);
  });
}

FMD_API fmd_status fmd_batch_rg(fmd_batch* b, int32_t slot, double* rg) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!rg) throw fmd::Error(FMD_ERR_ARG, "null rg");
    *rg = bb.rg(slot);
  });
}

FMD_API fmd_status fmd_batch_compute_forces(fmd_batch* b, int32_t slot, double* f, double* pe, double* virial) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    bb.forces(slot, f, pe, virial);
  });
}

FMD_API fmd_status fmd_batch_get_force_frame(fmd_batch* b, int32_t slot, double* xyz, double* box_L) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    bb.force_frame(slot, xyz, box_L);
  });
}

FMD_API fmd_status fmd_batch_stress_acf(fmd_batch* b, int32_t slot, int64_t* lag_steps, double* values,
                                        int64_t* counts, int32_t cap, int32_t* nrows) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!nrows || cap < 0 || (cap > 0 && (!lag_steps || !values || !counts))) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    std::vector<int64_t> lag, cnt;
    std::vector<double> val;
    bb.stress_acf(slot, lag, val, cnt);
    *nrows = (int32_t)lag.size();
    for (int32_t i = 0; i < cap && i < (int32_t)lag.size(); ++i) {
      lag_steps[i] = lag[i];
      counts[i] = cnt[i];
      for (int c = 0; c < 6; ++c) values[6 * i + c] = val[6 * (size_t)i + c];
    }
  });
}

FMD_API fmd_status fmd_batch_write_stress_acf(fmd_batch* b, int32_t slot, const char* path) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!path) throw fmd::Error(FMD_ERR_ARG, "null path");
    bb.write_stress_acf(slot, path);
  });
}

FMD_API fmd_status fmd_traj_write_batch(fmd_traj* t, fmd_batch* b, int32_t slot) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!t || !t->w) throw fmd::Error(FMD_ERR_ARG, "null trajectory");
    t->w->write(bb, slot);
  });
}

FMD_API fmd_status fmd_batch_pairs(fmd_batch* b, int32_t slot, int32_t* i, int32_t* j, int64_t cap, int64_t* n) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!n || (cap > 0 && (!i || !j))) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *n = bb.pairs(slot, i, j, cap);
  });
}

FMD_API fmd_status fmd_batch_totals(fmd_batch* b, int32_t* active, int64_t* atoms, int64_t* bytes) {
  return guarded([&] { B(b).totals(active, atoms, bytes); });
}

FMD_API fmd_status fmd_batch_mark(fmd_batch* b, int32_t which) {
  return guarded([&] { B(b).mark(which); });
}

FMD_API fmd_status fmd_batch_elapsed_ms(fmd_batch* b, double* ms) {
  return guarded([&] {
    if (!ms) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *ms = B(b).elapsed_ms();
  });
}

FMD_API fmd_status fmd_batch_time_force(fmd_batch* b, int32_t iters, double* ms) {
  return guarded([&] {
    if (!ms || iters <= 0) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    *ms = B(b).time_force(iters);
  });
}

FMD_API fmd_status fmd_batch_autotune(fmd_batch* b, int32_t iters, int32_t* chosen, double* ms_per_variant,
                                      int32_t cap) {
  return guarded([&] {
    if (iters <= 0 || cap < 0) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    const int v = B(b).autotune(iters, ms_per_variant, cap);
    if (chosen) *chosen = v;
    // entries after the force variants: neighbor-list variant times (ms per
    // full rebuild), then the chosen neighbor variant
    if (ms_per_variant) {
      for (int k = 0; k < fmd::mixed::kNbrVariants && fmd::mixed::kForceVariants + k < cap; ++k)
        ms_per_variant[fmd::mixed::kForceVariants + k] = B(b).nbr_variant_ms()[k];
      const int at = fmd::mixed::kForceVariants + fmd::mixed::kNbrVariants;
      if (at < cap) ms_per_variant[at] = B(b).nbr_variant();
    }
  });
}

FMD_API fmd_status fmd_batch_list_stats(fmd_batch* b, int64_t* entries, int32_t* max_per_atom) {
  return guarded([&] { B(b).list_stats(entries, max_per_atom); });
}

FMD_API fmd_status fmd_batch_kernels_per_step(fmd_batch* b, int32_t* n) {
  return guarded([&] {
    B(b);
    if (!n) throw fmd::Error(FMD_ERR_ARG, "null argument");
    // k_pre, k_commit, 9 rebuild kernels (plan, bin, scan, scatter, cell sort,
    // permute, bonded tables, home plan, list), k_force x2, k_post, k_post_commit
    *n = 15;
  });
}

FMD_API fmd_status fmd_batch_launch_counts(fmd_batch* b, int64_t* counts, int32_t n) {
  return guarded([&] {
    if (!counts || n < 0) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    B(b).launch_counts(counts, n);
  });
}

FMD_API fmd_status fmd_batch_set_list_prune(fmd_batch* b, int32_t slot, double delta) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    bb.set_list_prune(slot, delta);
  });
}

FMD_API fmd_status fmd_batch_set_list_buffer(fmd_batch* b, int32_t slot, double skin) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    bb.set_list_buffer(slot, skin);
  });
}

FMD_API fmd_status fmd_batch_get_list_buffer(fmd_batch* b, int32_t slot, double* skin) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!skin) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    *skin = bb.rep(slot).skin;
  });
}

FMD_API fmd_status fmd_batch_set_rebuild_cadence(fmd_batch* b, int32_t slot, int32_t max_steps) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    bb.set_max_between(slot, max_steps);
  });
}

FMD_API fmd_status fmd_batch_set_variants(fmd_batch* b, int32_t force_variant, int32_t nbr_variant) {
  return guarded([&] { B(b).set_variants(force_variant, nbr_variant); });
}

FMD_API fmd_status fmd_batch_get_variants(fmd_batch* b, int32_t* force_variant, int32_t* nbr_variant,
                                          int32_t* n_force, int32_t* n_nbr) {
  return guarded([&] {
    auto& bb = B(b);
    if (force_variant) *force_variant = bb.force_variant();
    if (nbr_variant) *nbr_variant = bb.nbr_variant();
    if (n_force) *n_force = fmd::mixed::kForceVariants;
    if (n_nbr) *n_nbr = fmd::mixed::kNbrVariants;
  });
}

FMD_API fmd_status fmd_batch_last_forces(fmd_batch* b, int32_t slot, double* f) {
  return guarded([&] {
    auto& bb = B(b);
    need_slot(bb, slot);
    if (!f) throw fmd::Error(FMD_ERR_ARG, "null argument");
    bb.last_forces(slot, f);
  });
}

}  // extern "C"
