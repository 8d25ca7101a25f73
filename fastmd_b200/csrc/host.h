// Host-side types shared by the engines: errors, run configuration, topology.
#pragma once
#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fastmd.h"

namespace fmd {

struct Error : std::runtime_error {
  fmd_status code;
  Error(fmd_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

// One tabulated pair potential: a keyword section of a LAMMPS pair_style
// table file (io/table_parser.cpp:7-87).  Grid parameters in single
// precision exactly as the reference derives them; per point the force
// column (applied as F/r, as force/table.cu:92-96 does) and the energy.
struct PairTable {
  std::string file, keyword;
  float rmin = 0, rmax = 0, dr = 0, inv_dr = 0;
  int32_t npoints = 0;
  std::vector<float> r, f, e;
};

PairTable read_pair_table(const std::string& path, const std::string& keyword);

// Parsed run.conf (the key set of src/io/config.cpp:32-127).
struct RunConfig {
  int32_t natoms = 0;
  int32_t ntypes = 0;
  double rc = 0, skin = 0, dt = 0;
  int64_t nsteps = 0;
  int32_t dump_freq = 0;
  int32_t thermo_on = 0, thermo_freq = 0;
  std::string thermo_file;
  int32_t stress_on = 0, stress_freq = 0;
  std::string stress_file;
  int32_t rg_on = 0, rg_freq = 0;
  std::string rg_file;
  int32_t restart_freq = -1;
  std::string restart_file;
  int32_t ensemble = FMD_LANGEVIN;
  double T_start = 0, T_stop = 0, Tdamp = 0;
  double P_start = 0, P_stop = 0, Pdamp = 0;
  int32_t chain_length = 3;
  // nh_chain_carry 1: the chain's upper accelerations carried between half
  // steps (LAMMPS fix nh); 0, the default, is the reference's scheme.
  int32_t nh_chain_carry = 0;
  uint64_t seed = 0;  // SimParams is zero-initialized; nvt_langevin defaults it to 42 (config.cpp:11, 79-81)
  std::string data_file, coords_file, forces_dump_file;
  std::vector<double> lj;                   // [ntypes*ntypes*2] (eps, sig)
  std::vector<std::array<double, 4>> bond;  // k, R0, eps, sig
  std::vector<std::array<double, 2>> angle; // k_theta, theta0 (radians)
  std::vector<PairTable> tables;            // distinct (file, keyword) sections
  std::vector<int32_t> table_of;            // [ntypes*ntypes]: index into tables, -1: none
};

RunConfig parse_run_conf(const std::string& text);

// A system in data-file order (what a LAMMPS data file or the generator gives).
struct Topology {
  int32_t natoms = 0;
  int32_t ntypes = 1;
  double box_L = 0;
  std::vector<double> xyz;     // [3N]
  std::vector<double> vel;     // [3N]
  std::vector<int32_t> image;  // [3N]
  std::vector<int32_t> type;   // [N]
  std::vector<int32_t> mol;    // [N]
  std::vector<double> mass;    // [ntypes]
  std::vector<int32_t> bonds;  // [2B]
  std::vector<int32_t> bond_type;
  std::vector<int32_t> angles;  // [3A]
  std::vector<int32_t> angle_type;
  int32_t nbonds() const { return (int32_t)bond_type.size(); }
  int32_t nangles() const { return (int32_t)angle_type.size(); }
};

Topology read_lammps_data(const std::string& path);
// Restart / data file in the reference's layout (io/lammps_data.cpp:269-385:
// header, Masses, "Atoms # full" with image flags, Velocities, Bonds,
// Angles), FP64 values written with enough digits to read back exactly.
void write_lammps_data(const std::string& path, const Topology& t, int64_t step);
Topology read_xyz_coords(const std::string& path, double box_L);
Topology topology_from_desc(const fmd_system_desc& d);
Topology generate_melt(const fmd_melt_spec& spec);

// Check that topology and run.conf agree (types, bond / angle types); fills
// defaults for masses.  Throws Error(FMD_ERR_CONFIG) on mismatch.
void validate(const RunConfig& cfg, Topology& topo);

// Restart state sidecar ("<data file>.state"): the run state a LAMMPS data
// file does not carry (step counter, thermostat / barostat chain, box and
// reference volume, list settings), as "key v1 v2 ..." text lines with
// doubles written to 17 significant digits (exact round trip).
struct StateFile {
  std::vector<std::pair<std::string, std::vector<double>>> entries;
  void put(const std::string& key, std::vector<double> v) { entries.emplace_back(key, std::move(v)); }
  bool has(const std::string& key) const;
  const std::vector<double>& get(const std::string& key) const;  // throws Error(FMD_ERR_IO) when missing
  double get1(const std::string& key) const { return get(key).at(0); }
};
std::string state_path(const std::string& data_path);
void write_state_file(const std::string& path, const StateFile& s);
bool read_state_file(const std::string& path, StateFile& s);  // false when the file does not exist

// Load the atoms for a simulation from one of the sources.
Topology load_atoms(const RunConfig& cfg, const char* data_path, const fmd_system_desc* desc,
                    const fmd_melt_spec* gen);

// Sorted unique 1-2 bonded partners per atom (lammps_data.cpp:231-253).
void build_exclusions(const Topology& t, std::vector<int32_t>& off, std::vector<int32_t>& list);

// Maximum neighbors per atom for a Verlet list (verlet_list.cu:4-7 formula).
int32_t reference_max_neighbors(int32_t natoms, double box_L, double rc_skin);

}  // namespace fmd
