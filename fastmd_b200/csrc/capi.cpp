// extern "C" entry points of include/fastmd.h for the host helpers and the
// one-system API.  Every call converts exceptions into a status code.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "engine.h"
#include "host.h"

namespace fmd {
const std::string& last_error();
}

struct fmd_sim {
  std::unique_ptr<fmd::SimEngine> eng;
  int32_t form = 0;
  fmd::Topology topo;  // topology and masses (the state lives in the engine)
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

void require_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw fmd::Error(FMD_ERR_NO_DEVICE, "no CUDA device available");
  }
}

}  // namespace

extern "C" {

FMD_API const char* fmd_version(void) { return "fastmd_b200 0.1.0 (sm_100a)"; }

FMD_API int32_t fmd_last_error(char* buf, size_t len) {
  const std::string& s = fmd::last_error();
  if (buf && len > 0) {
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  return (int32_t)s.size();
}

FMD_API fmd_status fmd_device_count(int32_t* n) {
  return guarded([&] {
    if (!n) throw fmd::Error(FMD_ERR_ARG, "null");
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
      cudaGetLastError();
      c = 0;
    }
    *n = c;
  });
}

FMD_API fmd_status fmd_generate_melt(const fmd_melt_spec* spec, int32_t* counts, double* box_L, double* xyz,
                                     int32_t* image, int32_t* type, int32_t* mol, int32_t* bonds, int32_t* angles) {
  return guarded([&] {
    if (!spec || !counts || !box_L) throw fmd::Error(FMD_ERR_ARG, "null argument");
    if (!xyz) {
      const int64_t n = (int64_t)spec->nchains * spec->chain_length;
      counts[0] = (int32_t)n;
      counts[1] = spec->nchains * std::max(0, spec->chain_length - 1);
      counts[2] = spec->nchains * std::max(0, spec->chain_length - 2);
      *box_L = std::cbrt((double)n / spec->density);
      return;
    }
    fmd::Topology t = fmd::generate_melt(*spec);
    counts[0] = t.natoms;
    counts[1] = t.nbonds();
    counts[2] = t.nangles();
    *box_L = t.box_L;
    std::memcpy(xyz, t.xyz.data(), t.xyz.size() * sizeof(double));
    if (image) std::memcpy(image, t.image.data(), t.image.size() * sizeof(int32_t));
    if (type) std::memcpy(type, t.type.data(), t.type.size() * sizeof(int32_t));
    if (mol) std::memcpy(mol, t.mol.data(), t.mol.size() * sizeof(int32_t));
    if (bonds) std::memcpy(bonds, t.bonds.data(), t.bonds.size() * sizeof(int32_t));
    if (angles) std::memcpy(angles, t.angles.data(), t.angles.size() * sizeof(int32_t));
  });
}

FMD_API fmd_status fmd_parse_run_conf(const char* text, int32_t* iout, double* fout, double* lj, int32_t lj_cap,
                                      double* bond, int32_t bond_cap, double* angle, int32_t angle_cap,
                                      uint64_t* seed) {
  return guarded([&] {
    if (!text || !iout || !fout) throw fmd::Error(FMD_ERR_ARG, "null argument");
    fmd::RunConfig c = fmd::parse_run_conf(text);
    const int32_t iv[11] = {c.natoms,  c.ntypes, (int32_t)c.nsteps, c.ensemble, c.chain_length, c.thermo_on,
                            c.thermo_freq, c.rg_on, c.rg_freq, (int32_t)c.bond.size(), (int32_t)c.angle.size()};
    std::memcpy(iout, iv, sizeof(iv));
    const double fv[9] = {c.rc, c.skin, c.dt, c.T_start, c.T_stop, c.Tdamp, c.P_start, c.P_stop, c.Pdamp};
    std::memcpy(fout, fv, sizeof(fv));
    if (lj)
      for (int k = 0; k < (int)c.lj.size() && k < lj_cap; ++k) lj[k] = c.lj[k];
    if (bond)
      for (int k = 0; k < (int)c.bond.size() && 4 * k + 3 < bond_cap; ++k)
        for (int e = 0; e < 4; ++e) bond[4 * k + e] = c.bond[k][e];
    if (angle)
      for (int k = 0; k < (int)c.angle.size() && 2 * k + 1 < angle_cap; ++k)
        for (int e = 0; e < 2; ++e) angle[2 * k + e] = c.angle[k][e];
    if (seed) *seed = c.seed;
  });
}

FMD_API fmd_status fmd_run_conf_outputs(const char* text, fmd_output_spec* out) {
  return guarded([&] {
    if (!text || !out) throw fmd::Error(FMD_ERR_ARG, "null argument");
    const fmd::RunConfig c = fmd::parse_run_conf(text);
    fmd_output_spec o{};
    o.nsteps = c.nsteps;
    o.ensemble = c.ensemble;
    o.thermo_on = c.thermo_on;
    o.thermo_freq = c.thermo_freq;
    o.rg_on = c.rg_on;
    o.rg_freq = c.rg_freq;
    o.stress_on = c.stress_on;
    o.stress_freq = c.stress_freq;
    o.dump_freq = c.dump_freq;
    o.restart_freq = c.restart_freq;
    auto put = [](char* dst, const std::string& v) {
      std::snprintf(dst, 256, "%s", v.c_str());
    };
    put(o.thermo_file, c.thermo_file);
    put(o.rg_file, c.rg_file);
    put(o.stress_file, c.stress_file);
    put(o.restart_file, c.restart_file);
    put(o.data_file, c.data_file);
    put(o.forces_dump_file, c.forces_dump_file);
    *out = o;
  });
}

FMD_API fmd_status fmd_restart_filename(const char* base, int64_t step, char* buf, size_t len) {
  return guarded([&] {
    if (!base || !buf || len == 0) throw fmd::Error(FMD_ERR_ARG, "null argument");
    const std::string b(base);
    const std::string tag = step >= 0 ? "_" + std::to_string(step) : std::string("_final");
    const size_t dot = b.rfind('.');
    const std::string name = dot != std::string::npos ? b.substr(0, dot) + tag + b.substr(dot) : b + tag;
    if (name.size() + 1 > len) throw fmd::Error(FMD_ERR_ARG, "buffer too small");
    std::memcpy(buf, name.c_str(), name.size() + 1);
  });
}

FMD_API fmd_status fmd_read_pair_table(const char* path, const char* keyword, float* grid, int32_t* npoints,
                                       float* data, int32_t cap) {
  return guarded([&] {
    if (!path || !keyword || !grid || !npoints || cap < 0 || (cap > 0 && !data))
      throw fmd::Error(FMD_ERR_ARG, "bad argument");
    const fmd::PairTable t = fmd::read_pair_table(path, keyword);
    grid[0] = t.rmin;
    grid[1] = t.rmax;
    grid[2] = t.dr;
    grid[3] = t.inv_dr;
    *npoints = t.npoints;
    for (int32_t k = 0; k < t.npoints && k < cap; ++k) {
      data[3 * k] = t.r[k];
      data[3 * k + 1] = t.f[k];
      data[3 * k + 2] = t.e[k];
    }
  });
}

FMD_API fmd_status fmd_run_conf_tables(const char* text, int32_t* table_of, int32_t cap, int32_t* ntables) {
  return guarded([&] {
    if (!text || !ntables || cap < 0 || (cap > 0 && !table_of)) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    const fmd::RunConfig c = fmd::parse_run_conf(text);
    *ntables = (int32_t)c.tables.size();
    for (int32_t k = 0; k < (int32_t)c.table_of.size() && k < cap; ++k) table_of[k] = c.table_of[k];
  });
}

FMD_API fmd_status fmd_read_lammps_data(const char* path, int32_t* counts, double* box_L, double* xyz,
                                        int32_t* image, int32_t* type, int32_t* mol, double* vel, int32_t* bonds,
                                        int32_t* bond_type, int32_t* angles, int32_t* angle_type, double* masses) {
  return guarded([&] {
    if (!path || !counts || !box_L) throw fmd::Error(FMD_ERR_ARG, "null argument");
    fmd::Topology t = fmd::read_lammps_data(path);
    counts[0] = t.natoms;
    counts[1] = t.nbonds();
    counts[2] = t.nangles();
    counts[3] = t.ntypes;
    *box_L = t.box_L;
    if (!xyz) return;
    std::memcpy(xyz, t.xyz.data(), t.xyz.size() * sizeof(double));
    if (image) std::memcpy(image, t.image.data(), t.image.size() * sizeof(int32_t));
    if (type) std::memcpy(type, t.type.data(), t.type.size() * sizeof(int32_t));
    if (mol) std::memcpy(mol, t.mol.data(), t.mol.size() * sizeof(int32_t));
    if (vel) std::memcpy(vel, t.vel.data(), t.vel.size() * sizeof(double));
    if (bonds) std::memcpy(bonds, t.bonds.data(), t.bonds.size() * sizeof(int32_t));
    if (bond_type) std::memcpy(bond_type, t.bond_type.data(), t.bond_type.size() * sizeof(int32_t));
    if (angles) std::memcpy(angles, t.angles.data(), t.angles.size() * sizeof(int32_t));
    if (angle_type) std::memcpy(angle_type, t.angle_type.data(), t.angle_type.size() * sizeof(int32_t));
    if (masses) std::memcpy(masses, t.mass.data(), t.mass.size() * sizeof(double));
  });
}

FMD_API fmd_status fmd_write_lammps_data(const char* path, const fmd_system_desc* desc, int64_t step) {
  return guarded([&] {
    if (!path || !desc) throw fmd::Error(FMD_ERR_ARG, "null argument");
    fmd::write_lammps_data(path, fmd::topology_from_desc(*desc), step);
  });
}

FMD_API fmd_status fmd_format_thermo_row(const fmd_thermo_row* r, char* buf, size_t len) {
  return guarded([&] {
    if (!r || !buf) throw fmd::Error(FMD_ERR_ARG, "null argument");
    std::snprintf(buf, len, "%d  %.4f  %.4f  %.4f  %.4f  %.4f  %.4f  %.4f  %.4f  %.4f", (int)r->step, r->ke, r->pe,
                  r->temp, r->stress[0], r->stress[1], r->stress[2], r->stress[3], r->stress[4], r->stress[5]);
  });
}

FMD_API fmd_status fmd_format_rg_row(int64_t step, double rg, char* buf, size_t len) {
  return guarded([&] {
    if (!buf) throw fmd::Error(FMD_ERR_ARG, "null argument");
    std::snprintf(buf, len, "%d  %.4f", (int)step, rg);
  });
}

FMD_API fmd_status fmd_sim_create(const char* conf, const char* data_path, const fmd_system_desc* desc,
                                  const fmd_melt_spec* gen, int32_t form, fmd_sim** out) {
  return guarded([&] {
    if (!conf || !out) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *out = nullptr;
    fmd::RunConfig cfg = fmd::parse_run_conf(conf);
    fmd::Topology t = fmd::load_atoms(cfg, data_path, desc, gen);
    require_device();
    std::unique_ptr<fmd_sim> s(new fmd_sim());
    s->form = form;
    s->topo = t;
    s->topo.xyz.clear();
    s->topo.vel.clear();
    s->topo.image.clear();
    // a data file written by fmd_write_restart carries a state sidecar: resume from it
    const std::string data = data_path ? std::string(data_path) : (desc || gen ? std::string() : cfg.data_file);
    fmd::StateFile st;
    const bool resume = !data.empty() && fmd::read_state_file(fmd::state_path(data), st);
    fmd::Topology saved;
    if (resume) saved = t;
    if (form == FMD_FORM_PLAIN_FP64)
      s->eng = fmd::make_plain_engine(cfg, std::move(t), gen);
    else if (form == FMD_FORM_MIXED)
      s->eng = fmd::make_mixed_engine(cfg, std::move(t), gen);
    else
      throw fmd::Error(FMD_ERR_ARG, "unknown form");
    if (resume) s->eng->restore(saved, st);
    *out = s.release();
  });
}

FMD_API fmd_status fmd_sim_destroy(fmd_sim* sim) {
  return guarded([&] { delete sim; });
}

#define SIM_CHECK() \
  if (!sim || !sim->eng) throw fmd::Error(FMD_ERR_ARG, "null simulation handle")

FMD_API fmd_status fmd_sim_info(const fmd_sim* sim, int32_t* natoms, int32_t* nbonds, int32_t* nangles, int64_t* step,
                                double* box_L) {
  return guarded([&] {
    SIM_CHECK();
    if (natoms) *natoms = sim->eng->natoms();
    if (nbonds) *nbonds = sim->eng->nbonds();
    if (nangles) *nangles = sim->eng->nangles();
    if (step) *step = sim->eng->step_count();
    if (box_L) *box_L = sim->eng->box_L();
  });
}

FMD_API fmd_status fmd_step(fmd_sim* sim, int64_t nsteps) {
  return guarded([&] {
    SIM_CHECK();
    if (nsteps < 0) throw fmd::Error(FMD_ERR_ARG, "nsteps < 0");
    sim->eng->step(nsteps);
  });
}

FMD_API fmd_status fmd_compute_forces(fmd_sim* sim, double* f, double* pe, double* virial) {
  return guarded([&] {
    SIM_CHECK();
    sim->eng->compute_forces(f, pe, virial);
  });
}

FMD_API fmd_status fmd_get_state(fmd_sim* sim, double* xyz, double* vel, int32_t* image) {
  return guarded([&] {
    SIM_CHECK();
    sim->eng->get_state(xyz, vel, image);
  });
}

FMD_API fmd_status fmd_set_state(fmd_sim* sim, const double* xyz, const double* vel, const int32_t* image) {
  return guarded([&] {
    SIM_CHECK();
    sim->eng->set_state(xyz, vel, image);
  });
}

FMD_API fmd_status fmd_stress_acf(fmd_sim* sim, int64_t* lag_steps, double* values, int64_t* counts, int32_t cap,
                                  int32_t* nrows) {
  return guarded([&] {
    SIM_CHECK();
    if (!nrows || cap < 0 || (cap > 0 && (!lag_steps || !values || !counts))) throw fmd::Error(FMD_ERR_ARG, "bad argument");
    std::vector<int64_t> lag, cnt;
    std::vector<double> val;
    sim->eng->stress_acf(lag, val, cnt);
    *nrows = (int32_t)lag.size();
    for (int32_t i = 0; i < cap && i < (int32_t)lag.size(); ++i) {
      lag_steps[i] = lag[i];
      counts[i] = cnt[i];
      for (int c = 0; c < 6; ++c) values[6 * i + c] = val[6 * (size_t)i + c];
    }
  });
}

FMD_API fmd_status fmd_write_stress_acf(fmd_sim* sim, const char* path) {
  return guarded([&] {
    SIM_CHECK();
    if (!path) throw fmd::Error(FMD_ERR_ARG, "null path");
    sim->eng->write_stress_acf(path);
  });
}

FMD_API fmd_status fmd_traj_open(const char* path, int32_t natoms, int32_t ntypes, fmd_traj** out) {
  return guarded([&] {
    if (!path || !out) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *out = nullptr;
    std::unique_ptr<fmd_traj> t(new fmd_traj());
    t->w.reset(new fmd::TrajWriter(path, natoms, ntypes));
    *out = t.release();
  });
}

FMD_API fmd_status fmd_traj_write_sim(fmd_traj* t, fmd_sim* sim) {
  return guarded([&] {
    SIM_CHECK();
    if (!t || !t->w) throw fmd::Error(FMD_ERR_ARG, "null trajectory");
    if (sim->eng->natoms() != t->w->natoms()) throw fmd::Error(FMD_ERR_ARG, "natoms differs from the trajectory's");
    sim->eng->dump_frame(*t->w);
  });
}

FMD_API fmd_status fmd_traj_close(fmd_traj* t) {
  return guarded([&] {
    if (!t) return;
    std::unique_ptr<fmd_traj> own(t);
    if (own->w) own->w->close();
  });
}

FMD_API fmd_status fmd_write_restart(fmd_sim* sim, const char* path) {
  return guarded([&] {
    SIM_CHECK();
    if (!path) throw fmd::Error(FMD_ERR_ARG, "null path");
    fmd::Topology t = sim->topo;
    fmd::StateFile st;
    sim->eng->checkpoint(t, st);
    fmd::write_lammps_data(path, t, sim->eng->step_count());
    fmd::write_state_file(fmd::state_path(path), st);
  });
}

FMD_API fmd_status fmd_thermo(fmd_sim* sim, fmd_thermo_row* row) {
  return guarded([&] {
    SIM_CHECK();
    if (!row) throw fmd::Error(FMD_ERR_ARG, "null row");
    sim->eng->thermo(row);
  });
}

FMD_API fmd_status fmd_rg(fmd_sim* sim, double* rg) {
  return guarded([&] {
    SIM_CHECK();
    if (!rg) throw fmd::Error(FMD_ERR_ARG, "null rg");
    *rg = sim->eng->rg();
  });
}

FMD_API fmd_status fmd_pairs(fmd_sim* sim, int32_t* i, int32_t* j, int64_t cap, int64_t* n) {
  return guarded([&] {
    SIM_CHECK();
    if (!n || (cap > 0 && (!i || !j))) throw fmd::Error(FMD_ERR_ARG, "null argument");
    *n = sim->eng->pairs(i, j, cap);
  });
}

FMD_API fmd_status fmd_sim_counters(const fmd_sim* sim, int64_t* rebuilds, int32_t* status_word, int32_t* max_neighbors) {
  return guarded([&] {
    SIM_CHECK();
    if (rebuilds) *rebuilds = sim->eng->rebuilds();
    if (status_word) *status_word = sim->eng->status_word();
    if (max_neighbors) *max_neighbors = sim->eng->max_neighbors();
  });
}

}  // extern "C"
