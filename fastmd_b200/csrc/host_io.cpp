// run.conf parsing, LAMMPS data reading, xyz coordinates and the seeded melt
// generator.  Host-only code; no CUDA calls.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_map>

#include "counter_rng.h"
#include "host.h"

namespace fmd {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

// ---------------------------------------------------------------------------
// Pair table file section (io/table_parser.cpp:7-87): skip blank and '#'
// lines; the section starts at the line whose first word is the keyword; the
// next line holds "N n [R rlo rhi]"; then n lines "index r energy force".
// Without R the grid spans the first and last r.  r must increase.
// ---------------------------------------------------------------------------
PairTable read_pair_table(const std::string& path, const std::string& keyword) {
  std::ifstream in(path);
  if (!in) throw Error(FMD_ERR_IO, "cannot open table file: " + path);
  PairTable t;
  t.file = path;
  t.keyword = keyword;
  std::string line;
  bool found = false, has_r = false;
  int n = 0;
  float rlo = 0, rhi = 0;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    std::string first;
    iss >> first;
    if (first != keyword) continue;
    found = true;
    while (std::getline(in, line)) {
      if (line.empty() || line[0] == '#') continue;
      std::istringstream hs(line);
      std::string key, rkey;
      hs >> key;
      if (key == "N") {
        hs >> n;
        if (hs >> rkey && rkey == "R") {
          hs >> rlo >> rhi;
          has_r = true;
        }
      }
      break;
    }
    break;
  }
  if (!found) throw Error(FMD_ERR_IO, "table keyword not found: " + keyword);
  if (n < 2) throw Error(FMD_ERR_IO, "table section " + keyword + " needs 'N n' with n >= 2");
  while ((int)t.r.size() < n && std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    int idx = 0;
    float r = 0, e = 0, f = 0;
    iss >> idx >> r >> e >> f;
    t.r.push_back(r);
    t.e.push_back(e);
    t.f.push_back(f);
  }
  if ((int)t.r.size() != n) throw Error(FMD_ERR_IO, "table data line count mismatch in " + path);
  for (int i = 1; i < n; ++i)
    if (!(t.r[i] > t.r[i - 1])) throw Error(FMD_ERR_IO, "table r values not monotonically increasing");
  if (!has_r) {
    rlo = t.r.front();
    rhi = t.r.back();
  }
  t.rmin = rlo;
  t.rmax = rhi;
  t.npoints = n;
  t.dr = (rhi - rlo) / (float)(n - 1);
  t.inv_dr = 1.0f / t.dr;
  return t;
}

// ---------------------------------------------------------------------------
// run.conf: whitespace-separated key/value lines, '#' comments, unknown keys
// ignored, deprecated keys rejected (src/io/config.cpp:10-213).
// ---------------------------------------------------------------------------
RunConfig parse_run_conf(const std::string& text) {
  RunConfig c;
  struct LJ {
    int ti, tj;
    double eps, sig;
  };
  std::vector<LJ> lj_entries;
  struct TableLine {
    int ti, tj;
    std::string file, keyword;
  };
  std::vector<TableLine> table_entries;
  std::istringstream in(text);
  std::string line;
  auto bad = [](const std::string& m) { throw Error(FMD_ERR_CONFIG, m); };
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    std::string key;
    iss >> key;
    if (key == "natoms") iss >> c.natoms;
    else if (key == "ntypes") iss >> c.ntypes;
    else if (key == "rc") iss >> c.rc;
    else if (key == "skin") iss >> c.skin;
    else if (key == "dt") iss >> c.dt;
    else if (key == "temperature")
      bad("'temperature' is deprecated. Use 'nvt_langevin T_start T_stop Tdamp [seed]' instead.");
    else if (key == "gamma")
      bad("'gamma' is deprecated. Use 'nvt_langevin T_start T_stop Tdamp [seed]' instead.");
    else if (key == "nsteps") iss >> c.nsteps;
    else if (key == "dump_freq") iss >> c.dump_freq;
    else if (key == "thermo") iss >> c.thermo_on >> c.thermo_freq >> c.thermo_file;
    else if (key == "stress") iss >> c.stress_on >> c.stress_freq >> c.stress_file;
    else if (key == "rg") iss >> c.rg_on >> c.rg_freq >> c.rg_file;
    else if (key == "restart") iss >> c.restart_freq >> c.restart_file;
    else if (key == "seed")
      bad("'seed' as a standalone key is deprecated. Specify seed in 'nvt_langevin T_start T_stop Tdamp [seed]'.");
    else if (key == "nvt_langevin") {
      c.ensemble = FMD_LANGEVIN;
      iss >> c.T_start >> c.T_stop >> c.Tdamp;
      unsigned long long s;
      if (iss >> s) c.seed = s;
      else c.seed = 42;
    } else if (key == "nvt_nh") {
      c.ensemble = FMD_NVT_NH;
      iss >> c.T_start >> c.T_stop >> c.Tdamp;
      if (!(iss >> c.chain_length)) c.chain_length = 3;
    } else if (key == "npt_nh") {
      c.ensemble = FMD_NPT_NH;
      iss >> c.T_start >> c.T_stop >> c.Tdamp >> c.P_start >> c.P_stop >> c.Pdamp;
      if (!(iss >> c.chain_length)) c.chain_length = 3;
    } else if (key == "nh_chain_carry") {
      iss >> c.nh_chain_carry;
      if (c.nh_chain_carry != 0 && c.nh_chain_carry != 1) bad("nh_chain_carry must be 0 or 1");
    } else if (key == "coords_file") iss >> c.coords_file;
    else if (key == "lammps_data_file") iss >> c.data_file;
    else if (key == "lj") {
      LJ e{};
      iss >> e.ti >> e.tj >> e.eps >> e.sig;
      lj_entries.push_back(e);
    } else if (key == "table") {
      TableLine e{};
      iss >> e.ti >> e.tj >> e.file >> e.keyword;
      table_entries.push_back(e);
    }
    else if (key == "bond_type") {
      int t = 0;
      double k = 0, R0 = 0, eps = 0, sig = 0;
      iss >> t >> k >> R0 >> eps >> sig;
      if (t < 0 || t > 1024) bad("bond_type index out of range");
      if ((int)c.bond.size() <= t) c.bond.resize(t + 1, {0, 0, 0, 0});
      c.bond[t] = {k, R0, eps, sig};
    } else if (key == "angle_type") {
      int t = 0;
      double k = 0, th = 0;
      iss >> t >> k >> th;
      if (t < 0 || t > 1024) bad("angle_type index out of range");
      if ((int)c.angle.size() <= t) c.angle.resize(t + 1, {0, 0});
      c.angle[t] = {k, th * 3.14159265358979323846 / 180.0};  // config.cpp:176
    } else if (key == "forces_dump_file") iss >> c.forces_dump_file;
  }
  if (c.ntypes < 1 || c.ntypes > 16) bad("ntypes must be in [1, 16]");
  c.lj.assign((size_t)c.ntypes * c.ntypes * 2, 0.0);
  for (auto& e : lj_entries) {  // config.cpp:130-134 (both orders)
    if (e.ti < 0 || e.ti >= c.ntypes || e.tj < 0 || e.tj >= c.ntypes) bad("lj type index out of range");
    c.lj[2 * (e.ti * c.ntypes + e.tj)] = e.eps;
    c.lj[2 * (e.ti * c.ntypes + e.tj) + 1] = e.sig;
    c.lj[2 * (e.tj * c.ntypes + e.ti)] = e.eps;
    c.lj[2 * (e.tj * c.ntypes + e.ti) + 1] = e.sig;
  }
  // config.cpp:136-162: one table per distinct (file, keyword), both orders;
  // a pair may not have both an lj and a table entry.
  c.table_of.assign((size_t)c.ntypes * c.ntypes, -1);
  for (auto& e : table_entries) {
    if (e.ti < 0 || e.ti >= c.ntypes || e.tj < 0 || e.tj >= c.ntypes) bad("table type index out of range");
    const size_t ij = (size_t)(e.ti * c.ntypes + e.tj);
    if (c.lj[2 * ij] != 0.0 || c.lj[2 * ij + 1] != 0.0)
      bad("Both lj and table defined for pair (" + std::to_string(e.ti) + "," + std::to_string(e.tj) + ")");
    int idx = -1;
    for (size_t k = 0; k < c.tables.size(); ++k)
      if (c.tables[k].file == e.file && c.tables[k].keyword == e.keyword) idx = (int)k;
    if (idx < 0) {
      c.tables.push_back(read_pair_table(e.file, e.keyword));
      idx = (int)c.tables.size() - 1;
    }
    c.table_of[ij] = idx;
    c.table_of[(size_t)(e.tj * c.ntypes + e.ti)] = idx;
  }
  // config.cpp:195-210
  if (c.ensemble == FMD_LANGEVIN && c.Tdamp <= 0) bad("Tdamp must be > 0 for nvt_langevin");
  if (c.ensemble != FMD_LANGEVIN) {
    if (c.Tdamp <= 0) bad("Tdamp must be > 0 for nvt_nh/npt_nh");
    if (c.chain_length < 1) bad("nh_chain_length must be >= 1");
    if (c.chain_length > 10) c.chain_length = 10;  // kMaxChainLength (nose_hoover.cuh:4, :313)
  }
  if (c.ensemble == FMD_NPT_NH && c.Pdamp <= 0) bad("Pdamp must be > 0 for npt_nh");
  if (c.rc <= 0) bad("rc must be > 0");
  if (c.skin < 0) bad("skin must be >= 0");
  if (c.dt <= 0) bad("dt must be > 0");
  return c;
}

// ---------------------------------------------------------------------------
// LAMMPS data file (src/io/lammps_data.cpp:18-229): cubic boxes, atom styles
// atomic / molecular / full / charge, optional image flags, Masses,
// Velocities, Bonds, Angles; 1-based ids and types made 0-based.
// ---------------------------------------------------------------------------
static std::vector<std::string> tokens(const std::string& s) {
  std::vector<std::string> t;
  std::istringstream iss(s);
  std::string w;
  while (iss >> w) t.push_back(w);
  return t;
}

Topology read_lammps_data(const std::string& path) {
  std::ifstream file(path);
  if (!file.is_open()) throw Error(FMD_ERR_IO, "Cannot open LAMMPS data file: " + path);
  std::vector<std::string> lines;
  for (std::string l; std::getline(file, l);) lines.push_back(l);
  double Lx = 0, Ly = 0, Lz = 0;
  int box_count = 0;
  for (const auto& line : lines) {
    if (box_count >= 3) break;
    size_t st = line.find_first_not_of(" \t\r\n");
    if (st == std::string::npos || line[st] == '#') continue;
    double lo, hi;
    char lab[8] = {0};
    if (std::sscanf(line.c_str() + st, "%lf %lf %3s", &lo, &hi, lab) == 3) {
      std::string label(lab);
      if (label == "xlo") { Lx = hi - lo; ++box_count; }
      else if (label == "ylo") { Ly = hi - lo; ++box_count; }
      else if (label == "zlo") { Lz = hi - lo; ++box_count; }
    }
  }
  if (box_count != 3) throw Error(FMD_ERR_IO, "LAMMPS data file missing box dimensions");
  if (std::fabs(Lx - Ly) > 1e-6 || std::fabs(Lx - Lz) > 1e-6)
    throw Error(FMD_ERR_IO, "Non-cubic box not supported");
  Topology t;
  t.box_L = Lx;
  enum Sec { None, Atoms, Vel, Bonds, Angles, Masses } cur = None;
  std::string style = "atomic";
  std::unordered_map<long long, int32_t> id2idx;
  std::vector<std::array<double, 3>> vels;
  std::vector<long long> vel_ids;
  std::vector<std::array<long long, 3>> raw_bonds;   // type, a, b
  std::vector<std::array<long long, 4>> raw_angles;  // type, a, b, c
  std::vector<double> masses;
  for (const auto& line : lines) {
    size_t st = line.find_first_not_of(" \t\r\n");
    if (st == std::string::npos) continue;
    std::string tr = line.substr(st);
    if (tr[0] == '#') continue;
    if (std::isupper((unsigned char)tr[0])) {
      cur = None;
      if (tr.rfind("Atoms", 0) == 0) {
        cur = Atoms;
        size_t h = tr.find('#');
        if (h != std::string::npos) {
          auto tk = tokens(tr.substr(h + 1));
          if (!tk.empty()) style = tk[0];
        }
      } else if (tr.rfind("Velocities", 0) == 0) cur = Vel;
      else if (tr.rfind("Bonds", 0) == 0) cur = Bonds;
      else if (tr.rfind("Angles", 0) == 0) cur = Angles;
      else if (tr.rfind("Masses", 0) == 0) cur = Masses;
      continue;
    }
    if (cur == None) continue;
    auto tk = tokens(tr);
    try {
      if (cur == Atoms) {
        size_t need, xo, io;
        long long mol = 1;
        if (style == "atomic") { need = 5; xo = 2; io = 5; }
        else if (style == "molecular") { need = 6; xo = 3; io = 6; }
        else if (style == "full" || style == "charge") { need = 7; xo = 4; io = 7; }
        else { need = 6; xo = 3; io = 6; }
        if (tk.size() < need) continue;
        long long id = std::stoll(tk[0]);
        int type;
        if (style == "atomic") type = std::stoi(tk[1]);
        else {
          mol = std::stoll(tk[1]);
          type = std::stoi(tk[2]);
        }
        int32_t idx = t.natoms++;
        id2idx[id] = idx;
        t.mol.push_back((int32_t)mol);
        t.type.push_back(type - 1);
        for (int d = 0; d < 3; ++d) t.xyz.push_back(std::stod(tk[xo + d]));
        for (int d = 0; d < 3; ++d) t.image.push_back(tk.size() >= io + 3 ? std::stoi(tk[io + d]) : 0);
      } else if (cur == Vel) {
        if (tk.size() < 4) continue;
        vel_ids.push_back(std::stoll(tk[0]));
        vels.push_back({std::stod(tk[1]), std::stod(tk[2]), std::stod(tk[3])});
      } else if (cur == Masses) {
        if (tk.size() < 2) continue;
        int tid = std::stoi(tk[0]);
        double m = std::stod(tk[1]);
        if (m <= 0) throw Error(FMD_ERR_IO, "mass must be > 0 for type " + std::to_string(tid));
        if (tid < 1) continue;
        if ((int)masses.size() < tid) masses.resize(tid, 1.0);
        masses[tid - 1] = m;
      } else if (cur == Bonds) {
        if (tk.size() < 4) continue;
        raw_bonds.push_back({std::stoll(tk[1]), std::stoll(tk[2]), std::stoll(tk[3])});
      } else if (cur == Angles) {
        if (tk.size() < 5) continue;
        raw_angles.push_back({std::stoll(tk[1]), std::stoll(tk[2]), std::stoll(tk[3]), std::stoll(tk[4])});
      }
    } catch (const Error&) {
      throw;
    } catch (const std::exception&) {
      continue;  // malformed numeric field: the reference's stream parse skips the line
    }
  }
  t.vel.assign((size_t)3 * t.natoms, 0.0);
  for (size_t k = 0; k < vels.size(); ++k) {
    auto it = id2idx.find(vel_ids[k]);
    if (it == id2idx.end()) continue;
    for (int d = 0; d < 3; ++d) t.vel[3 * it->second + d] = vels[k][d];
  }
  for (auto& b : raw_bonds) {
    auto i1 = id2idx.find(b[1]), i2 = id2idx.find(b[2]);
    if (i1 == id2idx.end() || i2 == id2idx.end()) continue;
    t.bonds.push_back(i1->second);
    t.bonds.push_back(i2->second);
    t.bond_type.push_back((int32_t)b[0] - 1);
  }
  for (auto& a : raw_angles) {
    auto i1 = id2idx.find(a[1]), i2 = id2idx.find(a[2]), i3 = id2idx.find(a[3]);
    if (i1 == id2idx.end() || i2 == id2idx.end() || i3 == id2idx.end()) continue;
    t.angles.push_back(i1->second);
    t.angles.push_back(i2->second);
    t.angles.push_back(i3->second);
    t.angle_type.push_back((int32_t)a[0] - 1);
  }
  int nt = 1;
  for (int ty : t.type) nt = std::max(nt, ty + 1);
  t.ntypes = nt;
  masses.resize(nt, 1.0);
  t.mass = masses;
  return t;
}

// xyz coordinates (config.cpp:179-192): count line, comment line, then
// "element x y z"; every atom gets type 0.
Topology read_xyz_coords(const std::string& path, double box_L) {
  std::ifstream cf(path);
  if (!cf.is_open()) throw Error(FMD_ERR_IO, "Cannot open coords file: " + path);
  Topology t;
  int n = 0;
  cf >> n;
  std::string comment;
  std::getline(cf, comment);
  std::getline(cf, comment);
  t.natoms = n;
  t.box_L = box_L;
  for (int i = 0; i < n; ++i) {
    std::string el;
    double x, y, z;
    if (!(cf >> el >> x >> y >> z)) throw Error(FMD_ERR_IO, "short coords file: " + path);
    t.xyz.insert(t.xyz.end(), {x, y, z});
  }
  t.vel.assign(3 * n, 0.0);
  t.image.assign(3 * n, 0);
  t.type.assign(n, 0);
  t.mol.assign(n, 1);
  t.mass = {1.0};
  return t;
}

void write_lammps_data(const std::string& path, const Topology& t, int64_t step) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) throw Error(FMD_ERR_IO, "cannot open " + path + " for writing");
  int nbt = 0, nat = 0;
  for (int32_t b : t.bond_type) nbt = std::max(nbt, b + 1);
  for (int32_t a : t.angle_type) nat = std::max(nat, a + 1);
  const int nb = t.nbonds(), na = t.nangles(), n = t.natoms;
  std::fprintf(fp, "# Restart from step %lld\n", (long long)step);
  std::fprintf(fp, "%d atoms\n%d atom types\n", n, t.ntypes);
  if (nb > 0) std::fprintf(fp, "%d bonds\n%d bond types\n", nb, nbt);
  if (na > 0) std::fprintf(fp, "%d angles\n%d angle types\n", na, nat);
  // all three box lines carry the edge (the reference's writer drops it from
  // the zhi line, io/lammps_data.cpp:335)
  std::fprintf(fp, "\n0.0 %.17g xlo xhi\n0.0 %.17g ylo yhi\n0.0 %.17g zlo zhi\n\n", t.box_L, t.box_L, t.box_L);
  std::fprintf(fp, "Masses\n\n");
  for (int k = 0; k < t.ntypes; ++k)
    std::fprintf(fp, "%d %.17g\n", k + 1, k < (int)t.mass.size() ? t.mass[k] : 1.0);
  std::fprintf(fp, "\nAtoms # full\n\n");
  for (int i = 0; i < n; ++i) {
    const int mol = t.mol.empty() ? 1 : t.mol[i];
    const int ix = t.image.empty() ? 0 : t.image[3 * i], iy = t.image.empty() ? 0 : t.image[3 * i + 1],
              iz = t.image.empty() ? 0 : t.image[3 * i + 2];
    std::fprintf(fp, "%d %d %d 0.0 %.17g %.17g %.17g %d %d %d\n", i + 1, mol, t.type[i] + 1, t.xyz[3 * i],
                 t.xyz[3 * i + 1], t.xyz[3 * i + 2], ix, iy, iz);
  }
  std::fprintf(fp, "\nVelocities\n\n");
  for (int i = 0; i < n; ++i) {
    const double vx = t.vel.empty() ? 0.0 : t.vel[3 * i], vy = t.vel.empty() ? 0.0 : t.vel[3 * i + 1],
                 vz = t.vel.empty() ? 0.0 : t.vel[3 * i + 2];
    std::fprintf(fp, "%d %.17g %.17g %.17g\n", i + 1, vx, vy, vz);
  }
  if (nb > 0) {
    std::fprintf(fp, "\nBonds\n\n");
    for (int b = 0; b < nb; ++b)
      std::fprintf(fp, "%d %d %d %d\n", b + 1, t.bond_type[b] + 1, t.bonds[2 * b] + 1, t.bonds[2 * b + 1] + 1);
  }
  if (na > 0) {
    std::fprintf(fp, "\nAngles\n\n");
    for (int a = 0; a < na; ++a)
      std::fprintf(fp, "%d %d %d %d %d\n", a + 1, t.angle_type[a] + 1, t.angles[3 * a] + 1, t.angles[3 * a + 1] + 1,
                   t.angles[3 * a + 2] + 1);
  }
  const bool bad = std::ferror(fp) != 0;
  if (std::fclose(fp) != 0 || bad) throw Error(FMD_ERR_IO, "write failed: " + path);
}

Topology topology_from_desc(const fmd_system_desc& d) {
  if (d.natoms <= 0 || !d.xyz || !d.type || d.box_L <= 0) throw Error(FMD_ERR_ARG, "system descriptor incomplete");
  Topology t;
  const int32_t n = d.natoms;
  t.natoms = n;
  t.box_L = d.box_L;
  t.xyz.assign(d.xyz, d.xyz + 3 * n);
  t.vel = d.vel ? std::vector<double>(d.vel, d.vel + 3 * n) : std::vector<double>(3 * n, 0.0);
  t.image = d.image ? std::vector<int32_t>(d.image, d.image + 3 * n) : std::vector<int32_t>(3 * n, 0);
  t.type.assign(d.type, d.type + n);
  t.mol = d.mol ? std::vector<int32_t>(d.mol, d.mol + n) : std::vector<int32_t>(n, 1);
  int nt = std::max(1, d.ntypes);
  for (int ty : t.type) nt = std::max(nt, ty + 1);
  t.ntypes = nt;
  t.mass.assign(nt, 1.0);
  if (d.mass)
    for (int k = 0; k < std::min(nt, d.ntypes); ++k) t.mass[k] = d.mass[k];
  if (d.nbonds > 0) {
    if (!d.bonds) throw Error(FMD_ERR_ARG, "bonds missing");
    t.bonds.assign(d.bonds, d.bonds + 2 * d.nbonds);
    t.bond_type = d.bond_type ? std::vector<int32_t>(d.bond_type, d.bond_type + d.nbonds)
                              : std::vector<int32_t>(d.nbonds, 0);
  }
  if (d.nangles > 0) {
    if (!d.angles) throw Error(FMD_ERR_ARG, "angles missing");
    t.angles.assign(d.angles, d.angles + 3 * d.nangles);
    t.angle_type = d.angle_type ? std::vector<int32_t>(d.angle_type, d.angle_type + d.nangles)
                                : std::vector<int32_t>(d.nangles, 0);
  }
  return t;
}

// ---------------------------------------------------------------------------
// Seeded Kremer-Grest melt.  Chains are random walks of step bond_length; a
// bead is placed at the first of up to 200 trial positions that is at least
// min_dist from every non-bonded bead already placed (the best trial when none
// is).  Chain starts are uniform in the box.  Draws: Philox stream GENW keyed
// on the seed, counter (bead index, trial).
// ---------------------------------------------------------------------------
Topology generate_melt(const fmd_melt_spec& sp) {
  if (sp.nchains <= 0 || sp.chain_length <= 0 || sp.density <= 0)
    throw Error(FMD_ERR_ARG, "melt spec needs nchains, chain_length, density > 0");
  const int64_t N64 = (int64_t)sp.nchains * sp.chain_length;
  if (N64 > (1ll << 30)) throw Error(FMD_ERR_ARG, "melt too large");
  const int32_t N = (int32_t)N64;
  const double bl = sp.bond_length > 0 ? sp.bond_length : 0.97;
  const double dmin = sp.min_dist > 0 ? sp.min_dist : 0.8;
  const double L = std::cbrt((double)N / sp.density);
  Topology t;
  t.natoms = N;
  t.box_L = L;
  t.xyz.resize(3 * (size_t)N);
  t.image.resize(3 * (size_t)N);
  t.vel.assign(3 * (size_t)N, 0.0);
  t.type.resize(N);
  t.mol.resize(N);
  // Rejection grid: cells of edge >= dmin.
  const int G = std::max(1, (int)std::floor(L / dmin));
  const double h = L / G;
  std::vector<int32_t> head((size_t)G * G * G, -1), next(N, -1);
  auto cell_of = [&](const double* p) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int v = (int)std::floor(p[d] / h);
      c[d] = ((v % G) + G) % G;
    }
    return ((size_t)c[2] * G + c[1]) * G + c[0];
  };
  auto nearest2 = [&](const double* p, int32_t skip) {
    double best = 1e300;
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int v = (int)std::floor(p[d] / h);
      c[d] = ((v % G) + G) % G;
    }
    const int r = (G >= 3) ? 1 : 0;
    int span = std::min(G, 3);
    for (int dz = -r; dz < -r + span; ++dz)
      for (int dy = -r; dy < -r + span; ++dy)
        for (int dx = -r; dx < -r + span; ++dx) {
          int cx = ((c[0] + dx) % G + G) % G, cy = ((c[1] + dy) % G + G) % G, cz = ((c[2] + dz) % G + G) % G;
          for (int32_t j = head[((size_t)cz * G + cy) * G + cx]; j >= 0; j = next[j]) {
            if (j == skip) continue;
            double d2 = 0;
            for (int d = 0; d < 3; ++d) {
              double u = p[d] - t.xyz[3 * (size_t)j + d];
              u -= L * std::nearbyint(u / L);
              d2 += u * u;
            }
            best = std::min(best, d2);
          }
        }
    return best;
  };
  const double dmin2 = dmin * dmin;
  std::vector<double> unwrapped(3);
  for (int32_t c = 0; c < sp.nchains; ++c) {
    double prev[3] = {0, 0, 0};
    for (int32_t k = 0; k < sp.chain_length; ++k) {
      const int32_t i = c * sp.chain_length + k;
      double best_p[3] = {0, 0, 0}, best_d2 = -1;
      for (uint32_t trial = 0; trial < 200; ++trial) {
        U32x4 ctr = {(uint32_t)i, trial, 0u, kStreamGenWalk};
        U32x4 r = philox4x32_10(ctr, (uint32_t)sp.seed, (uint32_t)(sp.seed >> 32));
        double p[3];
        if (k == 0) {
          p[0] = rng_uniform53(r.x, r.y) * L;
          p[1] = rng_uniform53(r.z, r.w) * L;
          U32x4 r2 = philox4x32_10({(uint32_t)i, trial, 1u, kStreamGenWalk}, (uint32_t)sp.seed,
                                   (uint32_t)(sp.seed >> 32));
          p[2] = rng_uniform53(r2.x, r2.y) * L;
        } else {
          double g[3];
          rng_normal3(sp.seed, kStreamGenWalk, trial, (uint32_t)i, &g[0], &g[1], &g[2]);
          double nrm = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
          if (nrm < 1e-12) continue;
          for (int d = 0; d < 3; ++d) p[d] = prev[d] + bl * g[d] / nrm;
        }
        double w[3];
        for (int d = 0; d < 3; ++d) w[d] = p[d] - L * std::floor(p[d] / L);
        double d2 = nearest2(w, k > 0 ? i - 1 : -1);
        if (d2 > best_d2) {
          best_d2 = d2;
          for (int d = 0; d < 3; ++d) best_p[d] = p[d];
        }
        if (d2 >= dmin2) break;
      }
      for (int d = 0; d < 3; ++d) {
        prev[d] = best_p[d];
        double fl = std::floor(best_p[d] / L);
        double w = best_p[d] - L * fl;
        if (w >= L) w -= L;  // guard the rounding edge
        if (w < 0) w = 0;
        t.xyz[3 * (size_t)i + d] = w;
        t.image[3 * (size_t)i + d] = (int32_t)fl;
      }
      const size_t cc = cell_of(&t.xyz[3 * (size_t)i]);
      next[i] = head[cc];
      head[cc] = i;
      t.type[i] = sp.type_block > 0 ? (k / sp.type_block) % 2 : 0;
      t.mol[i] = c + 1;
      if (k > 0) {
        t.bonds.push_back(i - 1);
        t.bonds.push_back(i);
        t.bond_type.push_back(0);
      }
      if (k > 1) {
        t.angles.push_back(i - 2);
        t.angles.push_back(i - 1);
        t.angles.push_back(i);
        t.angle_type.push_back(0);
      }
    }
  }
  t.ntypes = sp.type_block > 0 ? 2 : 1;
  t.mass.assign(t.ntypes, 1.0);
  return t;
}

void validate(const RunConfig& cfg, Topology& t) {
  if (t.natoms <= 0) throw Error(FMD_ERR_CONFIG, "system has no atoms");
  // The reference sizes every array from run.conf natoms (main.cu:62-99) and
  // overruns them when the data file holds more atoms; here a given natoms
  // must match the system, and an absent one is taken from it.
  if (cfg.natoms > 0 && cfg.natoms != t.natoms)
    throw Error(FMD_ERR_CONFIG, "run.conf natoms " + std::to_string(cfg.natoms) + " does not match the system's " +
                                    std::to_string(t.natoms) + " atoms");
  if (t.box_L <= 0) throw Error(FMD_ERR_CONFIG, "box edge must be > 0");
  for (int ty : t.type)
    if (ty < 0 || ty >= cfg.ntypes) throw Error(FMD_ERR_CONFIG, "atom type outside run.conf ntypes");
  t.ntypes = cfg.ntypes;
  t.mass.resize(cfg.ntypes, 1.0);
  for (int b : t.bond_type)
    if (b < 0 || b >= (int)cfg.bond.size()) throw Error(FMD_ERR_CONFIG, "bond type has no bond_type line");
  for (int a : t.angle_type)
    if (a < 0 || a >= (int)cfg.angle.size()) throw Error(FMD_ERR_CONFIG, "angle type has no angle_type line");
  for (int32_t b = 0; b < t.nbonds(); ++b)
    for (int e = 0; e < 2; ++e)
      if (t.bonds[2 * b + e] < 0 || t.bonds[2 * b + e] >= t.natoms) throw Error(FMD_ERR_CONFIG, "bond atom index");
  for (int32_t a = 0; a < t.nangles(); ++a)
    for (int e = 0; e < 3; ++e)
      if (t.angles[3 * a + e] < 0 || t.angles[3 * a + e] >= t.natoms) throw Error(FMD_ERR_CONFIG, "angle atom index");
  if (2.0 * cfg.rc > t.box_L) throw Error(FMD_ERR_CONFIG, "box edge must be at least 2 rc");
  if ((int64_t)t.xyz.size() != 3ll * t.natoms) throw Error(FMD_ERR_CONFIG, "position count mismatch");
  t.vel.resize(3 * (size_t)t.natoms, 0.0);
  t.image.resize(3 * (size_t)t.natoms, 0);
  t.mol.resize(t.natoms, 1);
  // Wrap positions into [0, L), folding whole periods into the image flags
  // (the reference's first pre-force step does the same wrap, langevin.cu:77-88).
  const double L = t.box_L;
  for (size_t k = 0; k < t.xyz.size(); ++k) {
    double fl = std::floor(t.xyz[k] / L);
    if (fl != 0.0) {
      t.xyz[k] -= fl * L;
      t.image[k] += (int32_t)fl;
    }
    if (t.xyz[k] >= L) {  // rounding edge: x just below a multiple of L
      t.xyz[k] -= L;
      t.image[k] += 1;
    }
    if (t.xyz[k] < 0.0) t.xyz[k] = 0.0;
  }
}

Topology load_atoms(const RunConfig& cfg, const char* data_path, const fmd_system_desc* desc,
                    const fmd_melt_spec* gen) {
  int sources = (data_path != nullptr) + (desc != nullptr) + (gen != nullptr);
  if (sources > 1) throw Error(FMD_ERR_ARG, "give at most one of data_path, desc, gen");
  Topology t;
  if (data_path) t = read_lammps_data(data_path);
  else if (desc) t = topology_from_desc(*desc);
  else if (gen) t = generate_melt(*gen);
  else if (!cfg.data_file.empty()) t = read_lammps_data(cfg.data_file);
  else if (!cfg.coords_file.empty()) throw Error(FMD_ERR_CONFIG, "coords_file needs a box: pass a system descriptor");
  else throw Error(FMD_ERR_CONFIG, "no atoms: set lammps_data_file or pass data_path / desc / gen");
  validate(cfg, t);
  return t;
}

void build_exclusions(const Topology& t, std::vector<int32_t>& off, std::vector<int32_t>& list) {
  std::vector<std::vector<int32_t>> per(t.natoms);
  for (int32_t b = 0; b < t.nbonds(); ++b) {
    per[t.bonds[2 * b]].push_back(t.bonds[2 * b + 1]);
    per[t.bonds[2 * b + 1]].push_back(t.bonds[2 * b]);
  }
  off.assign(t.natoms + 1, 0);
  list.clear();
  for (int32_t i = 0; i < t.natoms; ++i) {
    auto& l = per[i];
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
    off[i] = (int32_t)list.size();
    list.insert(list.end(), l.begin(), l.end());
  }
  off[t.natoms] = (int32_t)list.size();
}

int32_t reference_max_neighbors(int32_t natoms, double box_L, double rcs) {
  double density = natoms / (box_L * box_L * box_L);
  double sphere = (4.0 / 3.0) * 3.14159265358979323846 * rcs * rcs * rcs;
  int est = (int)(density * sphere * 3.0);
  return std::max(256, est);
}

// ---------------------------------------------------------------------------
// Restart state sidecar.
// ---------------------------------------------------------------------------
bool StateFile::has(const std::string& key) const {
  for (const auto& e : entries)
    if (e.first == key) return true;
  return false;
}

const std::vector<double>& StateFile::get(const std::string& key) const {
  for (const auto& e : entries)
    if (e.first == key) return e.second;
  throw Error(FMD_ERR_IO, "restart state file lacks '" + key + "'");
}

std::string state_path(const std::string& data_path) { return data_path + ".state"; }

void write_state_file(const std::string& path, const StateFile& s) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) throw Error(FMD_ERR_IO, "cannot write " + path);
  std::fprintf(fp, "# fastmd_b200 restart state v1\n");
  for (const auto& e : s.entries) {
    std::fprintf(fp, "%s", e.first.c_str());
    for (double v : e.second) std::fprintf(fp, " %.17g", v);
    std::fprintf(fp, "\n");
  }
  const bool ok = std::fflush(fp) == 0;
  std::fclose(fp);
  if (!ok) throw Error(FMD_ERR_IO, "cannot write " + path);
}

bool read_state_file(const std::string& path, StateFile& s) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  s.entries.clear();
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    std::string key;
    iss >> key;
    std::vector<double> v;
    std::string tok;
    while (iss >> tok) {
      char* end = nullptr;
      const double x = std::strtod(tok.c_str(), &end);
      if (!end || *end) throw Error(FMD_ERR_IO, "bad value in " + path + ": " + tok);
      v.push_back(x);
    }
    s.put(key, std::move(v));
  }
  return true;
}

}  // namespace fmd
