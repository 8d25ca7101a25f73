// C wrappers over the reference's own CPU code, compiled from the read-only
// reference tree by oracle/Makefile into oracle/_ref/libfmdref.so.
//
// TEST INFRASTRUCTURE ONLY: used to pin the FP64 oracle and the library's
// parsers against the reference's implementation.  Wrapped code:
//   reference/cpu_reference.hpp:7-298    (PBC, Morton sort, brute-force forces)
//   src/integrate/nose_hoover.cu:309-447 (NoseHooverState::init, host nh_propagate_chain)
//   src/io/config.cpp:10-220             (run.conf parser)
//   src/io/lammps_data.cpp:18-253        (LAMMPS data reader, exclusions)
// No kernel in the reference is launched through this file.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
using std::max;
using std::min;

#include "core/types.cuh"
#include "reference/cpu_reference.hpp"
#include "integrate/nose_hoover.cuh"
#include "io/config.hpp"
#include "io/table_parser.hpp"
#include "io/lammps_data.hpp"

namespace {
std::vector<float4> to_f4(const float* xyz, const int32_t* type, int32_t n) {
  std::vector<float4> p(n);
  for (int32_t i = 0; i < n; ++i)
    p[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], pack_type_id(type ? type[i] : 0));
  return p;
}
}  // namespace

extern "C" {

float ref_min_image(float dr, float L, float inv_L) { return ref::min_image(dr, L, inv_L); }

uint32_t ref_morton3d(float x, float y, float z, float inv_L) { return ref::morton3d(x, y, z, inv_L); }

void ref_morton_sort(const float* xyz, int32_t n, float inv_L, int32_t* perm) {
  auto p = to_f4(xyz, nullptr, n);
  auto r = ref::morton_sort_ref(p, inv_L);
  for (int32_t i = 0; i < n; ++i) perm[i] = r[i];
}

// Forces in FP32 as the reference's oracle computes them (no clamps).
void ref_brute_force_lj(const float* xyz, const int32_t* type, int32_t n, const float* lj, int32_t ntypes,
                        float rc, float L, const int32_t* excl_off, const int32_t* excl_list,
                        float* f, float* pe, float* vir) {
  auto p = to_f4(xyz, type, n);
  std::vector<float2> params(ntypes * ntypes);
  for (int32_t k = 0; k < ntypes * ntypes; ++k) params[k] = make_float2(lj[2 * k], lj[2 * k + 1]);
  std::vector<int> eo, el;
  if (excl_off) {
    eo.assign(excl_off, excl_off + n + 1);
    el.assign(excl_list, excl_list + excl_off[n]);
  }
  auto r = ref::brute_force_lj(p, params, ntypes, rc, L, 1.0f / L, excl_off ? &eo : nullptr,
                               excl_off ? &el : nullptr);
  for (int32_t i = 0; i < n; ++i) {
    f[3 * i] = r.fx[i];
    f[3 * i + 1] = r.fy[i];
    f[3 * i + 2] = r.fz[i];
    pe[i] = r.pe[i];
  }
  for (int c = 0; c < 6; ++c) vir[c] = r.virial[c];
}

void ref_brute_force_fene(const float* xyz, int32_t n, const int32_t* bonds, const int32_t* btype,
                          int32_t nbonds, const float* fene, int32_t ntypes, float L, float* f,
                          float* pe, float* vir) {
  auto p = to_f4(xyz, nullptr, n);
  std::vector<int2> b(nbonds);
  std::vector<int> t(btype, btype + nbonds);
  for (int32_t k = 0; k < nbonds; ++k) b[k] = make_int2(bonds[2 * k], bonds[2 * k + 1]);
  std::vector<float> K(ntypes), R0(ntypes), E(ntypes), S(ntypes);
  for (int32_t k = 0; k < ntypes; ++k) {
    K[k] = fene[4 * k];
    R0[k] = fene[4 * k + 1];
    E[k] = fene[4 * k + 2];
    S[k] = fene[4 * k + 3];
  }
  auto r = ref::brute_force_fene(p, b, t, K, R0, E, S, L, 1.0f / L);
  for (int32_t i = 0; i < n; ++i) {
    f[3 * i] = r.fx[i];
    f[3 * i + 1] = r.fy[i];
    f[3 * i + 2] = r.fz[i];
    pe[i] = r.pe[i];
  }
  for (int c = 0; c < 6; ++c) vir[c] = r.virial[c];
}

void ref_brute_force_angle(const float* xyz, int32_t n, const int32_t* angles, const int32_t* atype,
                           int32_t nangles, const float* ap, int32_t ntypes, float L, float* f,
                           float* pe, float* vir) {
  auto p = to_f4(xyz, nullptr, n);
  std::vector<int4> a(nangles);
  for (int32_t k = 0; k < nangles; ++k)
    a[k] = make_int4(angles[3 * k], angles[3 * k + 1], angles[3 * k + 2], atype[k]);
  std::vector<float> K(ntypes), T0(ntypes);
  for (int32_t k = 0; k < ntypes; ++k) {
    K[k] = ap[2 * k];
    T0[k] = ap[2 * k + 1];
  }
  auto r = ref::brute_force_angle(p, a, K, T0, L, 1.0f / L);
  for (int32_t i = 0; i < n; ++i) {
    f[3 * i] = r.fx[i];
    f[3 * i + 1] = r.fy[i];
    f[3 * i + 2] = r.fz[i];
    pe[i] = r.pe[i];
  }
  for (int c = 0; c < 6; ++c) vir[c] = r.virial[c];
}

// Unordered atom pairs (i < j) with ref::dist2_pbc(...) < rcs * rcs, the
// reference's FP32 pair predicate (cpu_reference.hpp:11-18), 1-2 bonded
// pairs given in excl CSR skipped.
int64_t ref_pairs_within(const float* xyz, int32_t n, float L, float rcs, const int32_t* excl_off,
                         const int32_t* excl_list, int32_t* pi, int32_t* pj, int64_t cap) {
  const float inv_L = 1.0f / L, rcs2 = rcs * rcs;
  int64_t m = 0;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = i + 1; j < n; ++j) {
      float d2 = ref::dist2_pbc(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], xyz[3 * j], xyz[3 * j + 1],
                                xyz[3 * j + 2], L, inv_L);
      if (!(d2 < rcs2)) continue;
      bool ex = false;
      if (excl_off)
        for (int32_t e = excl_off[i]; e < excl_off[i + 1]; ++e) ex |= (excl_list[e] == j);
      if (ex) continue;
      if (m < cap) {
        pi[m] = i;
        pj[m] = j;
      }
      ++m;
    }
  return m;
}

// Tile pairs within rc_skin (cpu_reference.hpp:59-87): out[2k], out[2k+1].
int64_t ref_brute_force_tile_list(const float* xyz, int32_t n, int32_t ntiles, float rcs, float L,
                                  int32_t* out, int64_t cap) {
  auto p = to_f4(xyz, nullptr, n);
  auto r = ref::brute_force_tile_list(p, ntiles, rcs, L, 1.0f / L);
  for (int64_t k = 0; k < (int64_t)r.size() && k < cap; ++k) {
    out[2 * k] = r[k].tile_a;
    out[2 * k + 1] = r[k].tile_b;
  }
  return (int64_t)r.size();
}

// One host chain half step from a given chain state (nose_hoover.cu:356-447).
void ref_nh_chain(int32_t natoms, float T, float Tdamp, int32_t M, float* xi, float* v_xi,
                  float total_KE, float half_dt, float* scale, float* Q) {
  SimParams params = {};
  params.natoms = natoms;
  params.box_L = 10.0f;
  params.inv_L = 0.1f;
  params.dt = 2.0f * half_dt;
  params.ensemble = Ensemble::NVT_NH;
  params.T_start = T;
  params.T_stop = T;
  params.Tdamp = Tdamp;
  params.nh_chain_length = M;
  NoseHooverState nh;
  nh.init(params);
  for (int k = 0; k < M; ++k) {
    nh.xi[k] = xi[k];
    nh.v_xi[k] = v_xi[k];
  }
  nh_propagate_chain(nh, total_KE, half_dt, *scale);
  for (int k = 0; k < M; ++k) {
    xi[k] = nh.xi[k];
    v_xi[k] = nh.v_xi[k];
  }
  Q[0] = nh.Q1;
  Q[1] = nh.Q_rest;
}

// run.conf parser (io/config.cpp).  fout: rc, skin, dt, T_start, T_stop, Tdamp,
// P_start, P_stop, Pdamp.  iout: natoms, ntypes, nsteps, ensemble, chain length,
// thermo_on, thermo_freq, rg_on, rg_freq, n_lj, n_bond_types, n_angle_types.
// lj [ntypes^2*2], bond [4*nbt], angle [2*nat] (theta0 radians), seed.
int32_t ref_parse_config(const char* path, float* fout, int32_t* iout, float* lj, int32_t lj_cap,
                         float* bond, int32_t bond_cap, float* angle, int32_t angle_cap,
                         uint64_t* seed, char* err, int32_t err_len) {
  try {
    TopologyData topo;
    SimParams p = parse_config(path, topo);
    fout[0] = p.rc;
    fout[1] = p.skin;
    fout[2] = p.dt;
    fout[3] = p.T_start;
    fout[4] = p.T_stop;
    fout[5] = p.Tdamp;
    fout[6] = p.P_start;
    fout[7] = p.P_stop;
    fout[8] = p.Pdamp;
    iout[0] = p.natoms;
    iout[1] = p.ntypes;
    iout[2] = p.nsteps;
    iout[3] = (int32_t)p.ensemble;
    iout[4] = p.nh_chain_length;
    iout[5] = p.thermo_on;
    iout[6] = p.thermo_freq;
    iout[7] = p.rg_on;
    iout[8] = p.rg_freq;
    iout[9] = (int32_t)topo.lj_params.size();
    iout[10] = (int32_t)topo.bond_params.size();
    iout[11] = (int32_t)topo.angle_params.size();
    for (int32_t k = 0; k < (int32_t)topo.lj_params.size() && 2 * k + 1 < lj_cap; ++k) {
      lj[2 * k] = topo.lj_params[k].x;
      lj[2 * k + 1] = topo.lj_params[k].y;
    }
    for (int32_t k = 0; k < (int32_t)topo.bond_params.size() && 4 * k + 3 < bond_cap; ++k) {
      bond[4 * k] = topo.bond_params[k].k;
      bond[4 * k + 1] = topo.bond_params[k].R0;
      bond[4 * k + 2] = topo.bond_params[k].eps;
      bond[4 * k + 3] = topo.bond_params[k].sig;
    }
    for (int32_t k = 0; k < (int32_t)topo.angle_params.size() && 2 * k + 1 < angle_cap; ++k) {
      angle[2 * k] = topo.angle_params[k].k_theta;
      angle[2 * k + 1] = topo.angle_params[k].theta0;
    }
    *seed = p.seed;
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return 1;
  }
}

// Pair table section reader (io/table_parser.cpp:7-87).  grid: rmin, rmax,
// dr, inv_dr; data: r, force, energy per point (cap points at most).
int32_t ref_parse_table(const char* path, const char* keyword, float* grid, int32_t* npoints, float* data,
                        int32_t cap, char* err, int32_t err_len) {
  try {
    TableFileData t = parse_table_file(path, keyword);
    grid[0] = t.params[0].rmin;
    grid[1] = t.params[0].rmax;
    grid[2] = t.params[0].dr;
    grid[3] = t.params[0].inv_dr;
    *npoints = t.params[0].npoints;
    for (int32_t k = 0; k < (int32_t)t.data.size() && k < cap; ++k) {
      data[3 * k] = t.data[k].x;
      data[3 * k + 1] = t.data[k].y;
      data[3 * k + 2] = t.data[k].z;
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return 1;
  }
}

// LAMMPS data reader (io/lammps_data.cpp:18-229).  counts: natoms, nbonds,
// nangles, nmasses.  Arrays sized by the caller from a first call with
// xyz == NULL (which fills counts only).
int32_t ref_parse_lammps_data(const char* path, int32_t* counts, float* box_L, float* xyz,
                              int32_t* type, int32_t* mol, int32_t* image, float* vel,
                              int32_t* bonds, int32_t* btype, int32_t* angles, int32_t* atype,
                              float* masses, char* err, int32_t err_len) {
  try {
    TopologyData topo;
    parse_lammps_data(path, topo);
    const int32_t n = (int32_t)topo.positions.size();
    counts[0] = n;
    counts[1] = (int32_t)topo.bonds.size();
    counts[2] = (int32_t)topo.angles.size();
    counts[3] = (int32_t)topo.masses.size();
    *box_L = topo.box_L;
    if (!xyz) return 0;
    for (int32_t i = 0; i < n; ++i) {
      xyz[3 * i] = topo.positions[i].x;
      xyz[3 * i + 1] = topo.positions[i].y;
      xyz[3 * i + 2] = topo.positions[i].z;
      type[i] = unpack_type_id(topo.positions[i].w);
      mol[i] = topo.mol_ids[i];
      for (int d = 0; d < 3; ++d) image[3 * i + d] = topo.images[3 * i + d];
      float4 v = (i < (int32_t)topo.velocities.size()) ? topo.velocities[i] : make_float4(0, 0, 0, 0);
      vel[3 * i] = v.x;
      vel[3 * i + 1] = v.y;
      vel[3 * i + 2] = v.z;
    }
    for (int32_t k = 0; k < counts[1]; ++k) {
      bonds[2 * k] = topo.bonds[k].x;
      bonds[2 * k + 1] = topo.bonds[k].y;
      btype[k] = topo.bond_types[k];
    }
    for (int32_t k = 0; k < counts[2]; ++k) {
      angles[3 * k] = topo.angles[k].x;
      angles[3 * k + 1] = topo.angles[k].y;
      angles[3 * k + 2] = topo.angles[k].z;
      atype[k] = topo.angles[k].w;
    }
    for (int32_t k = 0; k < counts[3]; ++k) masses[k] = topo.masses[k];
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return 1;
  }
}

}  // extern "C"
