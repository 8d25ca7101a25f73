// fastmd <run.conf> [--plain]: the process boundary of the reference
// (src/main.cu:24-36) as a thin program over the C ABI (include/fastmd.h).
//
// Reads the run.conf (src/io/config.cpp keys) and the LAMMPS data file it
// names, advances nsteps, and writes what the reference writes, when it
// writes it (src/main.cu:632-691, 738-783):
//   thermo  <on> <freq> <file>   "# step  KE  PE  T  Pxx  Pyy  Pzz  Pxy  Pxz  Pyz"
//                                then "%d  %.4f ..." rows (analysis/thermo.cu:80, 190-192)
//   rg      <on> <freq> <file>   "# step  Rg", "%d  %.4f" rows (analysis/rg.cu:95, 127-129)
//   restart <freq> <file>        LAMMPS data files <base>_<step><ext> every freq steps
//                                (not at the last step) and <base>_final<ext> at the end
//                                (io/lammps_data.cpp:255-267), each with a state sidecar
//   dump_freq <n>                traj.bin frames (io/dump.cu:12-56)
//   stress  <on> <freq> <file>   the stress autocorrelation rows at the end
//   forces_dump_file <file>      initial forces "# id fx fy fz pe" then exit
// and the reference's closing "Wall time: ... | Steps/s: ... | ns/day: ..." line.
// --plain runs the FP64 plain form instead of the mixed form.
//
// Errors: a message on stderr and exit status 1 (the reference throws
// std::runtime_error or exits through CUDA_CHECK); nothing else exits.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fastmd.h"

namespace {

struct Fail {
  std::string msg;
};

void check(fmd_status st, const char* what) {
  if (st == FMD_OK) return;
  char buf[1024] = {0};
  fmd_last_error(buf, sizeof(buf));
  throw Fail{std::string(what) + ": " + buf};
}

std::string read_text(const char* path) {
  std::ifstream in(path);
  if (!in) throw Fail{std::string("cannot open config file ") + path};
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

FILE* open_out(const char* path, const char* header) {
  FILE* fp = std::fopen(path, "w");
  if (!fp) throw Fail{std::string("cannot open output file ") + path};
  if (header) {
    std::fprintf(fp, "%s\n", header);
    std::fflush(fp);
  }
  return fp;
}

// Steps from `step` to the next multiple of freq (freq <= 0: never).
int64_t until(int64_t step, int64_t freq) {
  if (freq <= 0) return INT64_MAX;
  return freq - step % freq;
}

int run(int argc, char** argv) {
  const char* conf_path = nullptr;
  int32_t form = FMD_FORM_MIXED;
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--plain")) form = FMD_FORM_PLAIN_FP64;
    else if (argv[a][0] == '-' && argv[a][1] == '-') throw Fail{std::string("unknown option ") + argv[a]};
    else if (!conf_path) conf_path = argv[a];
    else throw Fail{"more than one config file given"};
  }
  if (!conf_path) {
    std::fprintf(stderr, "Usage: %s <config_file> [--plain]\n", argv[0]);
    return 1;
  }
  const std::string text = read_text(conf_path);
  fmd_output_spec out;
  check(fmd_run_conf_outputs(text.c_str(), &out), "config");
  int32_t iout[11];
  double fout[9];
  check(fmd_parse_run_conf(text.c_str(), iout, fout, nullptr, 0, nullptr, 0, nullptr, 0, nullptr), "config");
  const int32_t ntypes = iout[1];
  const double dt = fout[2];

  fmd_sim* sim = nullptr;
  check(fmd_sim_create(text.c_str(), nullptr, nullptr, nullptr, form, &sim), "setup");
  int32_t natoms = 0, nbonds = 0, nangles = 0;
  int64_t step0 = 0;
  double box = 0;
  check(fmd_sim_info(sim, &natoms, &nbonds, &nangles, &step0, &box), "setup");
  std::printf("[setup]  atoms=%d  box=%.2f  nsteps=%lld  form=%s", natoms, box, (long long)out.nsteps,
              form == FMD_FORM_MIXED ? "mixed" : "plain_fp64");
  if (nbonds > 0) std::printf("  bonds=%d", nbonds);
  if (nangles > 0) std::printf("  angles=%d", nangles);
  std::printf("\n\n");

  if (out.forces_dump_file[0]) {  // main.cu:344-362
    std::vector<double> f(3 * (size_t)natoms), pe(natoms);
    check(fmd_compute_forces(sim, f.data(), pe.data(), nullptr), "forces");
    FILE* fp = open_out(out.forces_dump_file, "# id fx fy fz pe");
    for (int i = 0; i < natoms; ++i)
      std::fprintf(fp, "%d %.6e %.6e %.6e %.6e\n", i, f[3 * i], f[3 * i + 1], f[3 * i + 2], pe[i]);
    std::fclose(fp);
    std::printf("Initial forces written to %s\n", out.forces_dump_file);
    fmd_sim_destroy(sim);
    return 0;
  }

  FILE* thermo = out.thermo_on ? open_out(out.thermo_file, "# step  KE  PE  T  Pxx  Pyy  Pzz  Pxy  Pxz  Pyz") : nullptr;
  FILE* rgf = out.rg_on ? open_out(out.rg_file, "# step  Rg") : nullptr;
  fmd_traj* traj = nullptr;
  if (out.dump_freq > 0) check(fmd_traj_open("traj.bin", natoms, ntypes, &traj), "dump");
  char line[512];

  const auto t0 = std::chrono::steady_clock::now();
  int64_t step = 0;
  const int64_t nsteps = out.nsteps;
  while (step < nsteps) {
    int64_t k = nsteps - step;
    if (out.thermo_on) k = std::min(k, until(step, out.thermo_freq));
    if (out.rg_on) k = std::min(k, until(step, out.rg_freq));
    k = std::min(k, until(step, out.dump_freq));
    k = std::min(k, until(step, out.restart_freq));
    check(fmd_step(sim, k), "step");
    step += k;
    if (out.thermo_on && out.thermo_freq > 0 && step % out.thermo_freq == 0) {
      fmd_thermo_row row;
      check(fmd_thermo(sim, &row), "thermo");
      check(fmd_format_thermo_row(&row, line, sizeof(line)), "thermo");
      std::fprintf(thermo, "%s\n", line);
      std::fflush(thermo);
      std::printf("Step %6lld  T=%10.4f  KE=%11.4f  PE=%11.4f  Etot=%11.4f  Pxx=%8.4f\n", (long long)step, row.temp,
                  row.ke, row.pe, row.ke + row.pe, row.stress[0]);
    }
    if (out.rg_on && out.rg_freq > 0 && step % out.rg_freq == 0) {
      double rg = 0;
      check(fmd_rg(sim, &rg), "rg");
      check(fmd_format_rg_row(step, rg, line, sizeof(line)), "rg");
      std::fprintf(rgf, "%s\n", line);
      std::fflush(rgf);
    }
    if (traj && step % out.dump_freq == 0) check(fmd_traj_write_sim(traj, sim), "dump");
    if (out.restart_freq > 0 && step % out.restart_freq == 0 && step != nsteps) {
      check(fmd_restart_filename(out.restart_file, step, line, sizeof(line)), "restart");
      check(fmd_write_restart(sim, line), "restart");
    }
  }
  if (out.restart_freq >= 0) {
    check(fmd_restart_filename(out.restart_file, -1, line, sizeof(line)), "restart");
    check(fmd_write_restart(sim, line), "restart");
  }
  const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const double sps = elapsed > 0 ? (double)nsteps / elapsed : 0.0;
  std::printf("Wall time: %.3f s  |  Steps/s: %.1f  |  ns/day: %.3f\n", elapsed, sps,
              elapsed > 0 ? ((double)nsteps * dt) / (elapsed / 86400.0) : 0.0);
  if (out.stress_on) {
    check(fmd_write_stress_acf(sim, out.stress_file), "stress");
    std::printf("Stress autocorrelation written to %s\n", out.stress_file);
  }
  if (traj) check(fmd_traj_close(traj), "dump");
  if (thermo) std::fclose(thermo);
  if (rgf) std::fclose(rgf);
  check(fmd_sim_destroy(sim), "teardown");
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const Fail& f) {
    std::fprintf(stderr, "Error: %s\n", f.msg.c_str());
    return 1;
  }
}
