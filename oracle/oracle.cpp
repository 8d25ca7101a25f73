// FP64 CPU oracle for the bead-spring MD per-step path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
// baseline.  The library never links or calls it.  See oracle.h for the list of
// reference files restated here; each function below cites the lines it follows.
// Built with -ffp-contract=off so every product and sum rounds exactly as
// written (no fused multiply-add), matching the library's FP64 plain kernels.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Counter RNG, restated from the library's specification (Philox4x32-10 and a
// Box-Muller transform with series log / sin / cos; see counter_rng.h there).
// ---------------------------------------------------------------------------
uint32_t mulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

void philox10(const uint32_t in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t a0 = 0xD2511F53u * c0, h0 = mulhi32(0xD2511F53u, c0);
    uint32_t a1 = 0xCD9E8D57u * c2, h1 = mulhi32(0xCD9E8D57u, c2);
    uint32_t n0 = h1 ^ c1 ^ k0, n2 = h0 ^ c3 ^ k1;
    c0 = n0;
    c1 = a1;
    c2 = n2;
    c3 = a0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

double series_log(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  int e = (int)((u >> 52) & 0x7FF) - 1023;
  u = (u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m;
  std::memcpy(&m, &u, 8);
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  double s = (m - 1.0) / (m + 1.0);
  double z = s * s;
  static const double inv_odd[11] = {1.0 / 23.0, 1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0,
                                     1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0, 1.0 / 9.0,
                                     1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0};
  double p = inv_odd[0];
  for (int k = 1; k < 11; ++k) p = std::fma(p, z, inv_odd[k]);
  double two_s = 2.0 * s;
  double lnm = std::fma(two_s * z, p, two_s);
  const double ln2_hi = 0x1.62e42f0000000p-1, ln2_lo = 0x1.df473de6af279p-26;
  double de = (double)e;
  return std::fma(de, ln2_hi, std::fma(de, ln2_lo, lnm));
}

void series_sincos_quarter(double g, double* s, double* c) {
  const double pio2_hi = 0x1.921fb50000000p+0, pio2_lo = 0x1.110b4611a6263p-26;
  double t = std::fma(g, pio2_hi, g * pio2_lo);
  double t2 = t * t;
  static const double sc[8] = {-1.0 / 355687428096000.0, 1.0 / 1307674368000.0,
                               -1.0 / 6227020800.0,      1.0 / 39916800.0,
                               -1.0 / 362880.0,          1.0 / 5040.0,
                               -1.0 / 120.0,             1.0 / 6.0};
  double ps = sc[0];
  for (int k = 1; k < 8; ++k) ps = std::fma(ps, t2, sc[k]);
  *s = std::fma(-(t * t2), ps, t);
  static const double cc[9] = {1.0 / 6402373705728000.0, -1.0 / 20922789888000.0,
                               1.0 / 87178291200.0,      -1.0 / 479001600.0,
                               1.0 / 3628800.0,          -1.0 / 40320.0,
                               1.0 / 720.0,              -1.0 / 24.0,
                               0.5};
  double pc = cc[0];
  for (int k = 1; k < 9; ++k) pc = std::fma(pc, t2, cc[k]);
  *c = std::fma(-t2, pc, 1.0);
}

void box_muller(uint32_t a, uint32_t b, double* z0, double* z1) {
  double u1 = ((double)a + 1.0) * 0x1.0p-32;
  double r = std::sqrt(-2.0 * series_log(u1));
  uint32_t q = b >> 30;
  double f = (double)(b & 0x3FFFFFFFu) * 0x1.0p-30;
  double s, c;
  if (f > 0.5)
    series_sincos_quarter(1.0 - f, &c, &s);
  else
    series_sincos_quarter(f, &s, &c);
  double cs, sn;
  if (q == 0) {
    cs = c;
    sn = s;
  } else if (q == 1) {
    cs = -s;
    sn = c;
  } else if (q == 2) {
    cs = -c;
    sn = -s;
  } else {
    cs = s;
    sn = -c;
  }
  *z0 = r * cs;
  *z1 = r * sn;
}

void normal3(uint64_t seed, uint32_t stream, uint64_t step, uint32_t id, double out[3]) {
  uint32_t c[4] = {id, (uint32_t)step, (uint32_t)(step >> 32), stream};
  uint32_t r[4];
  philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32), r);
  double z3;
  box_muller(r[0], r[1], &out[0], &out[1]);
  box_muller(r[2], r[3], &out[2], &z3);
}

const uint32_t kStreamLangevin = 0x4C414E47u;

// ---------------------------------------------------------------------------
// PBC (core/pbc.cuh:4-28) and displacement trigger (neighbor/skin_trigger.cuh:6-16)
// ---------------------------------------------------------------------------
inline double min_image(double dr, double L, double inv_L) { return dr - L * std::nearbyint(dr * inv_L); }
inline double round_image(double dr, double L, double inv_L) { return dr - L * std::round(dr * inv_L); }

// Exclusions: sorted unique 1-2 bonded partners per atom (io/lammps_data.cpp:231-253).
struct Excl {
  std::vector<int32_t> off, list;
  void build(int32_t n, const int32_t* bonds, int32_t nb) {
    std::vector<std::vector<int32_t>> per(n);
    for (int32_t b = 0; b < nb; ++b) {
      per[bonds[2 * b]].push_back(bonds[2 * b + 1]);
      per[bonds[2 * b + 1]].push_back(bonds[2 * b]);
    }
    off.assign(n + 1, 0);
    list.clear();
    for (int32_t i = 0; i < n; ++i) {
      auto& l = per[i];
      std::sort(l.begin(), l.end());
      l.erase(std::unique(l.begin(), l.end()), l.end());
      off[i] = (int32_t)list.size();
      list.insert(list.end(), l.begin(), l.end());
    }
    off[n] = (int32_t)list.size();
  }
  bool has(int32_t i, int32_t j) const {
    for (int32_t e = off[i]; e < off[i + 1]; ++e)
      if (list[e] == j) return true;
    return false;
  }
};

// ---------------------------------------------------------------------------
// Verlet list (neighbor/verlet_list.cu:3-13 grid, :58-75 binning, :82-104 cell
// ranges, :108-335 traversal).  The grid is re-derived from the current L at
// every build (the reference fixes it at allocation, verlet_list.cu:8-13).
// ---------------------------------------------------------------------------
struct Verlet {
  int32_t nx = 1, max_nbr = 0;
  std::vector<int32_t> nbr, cnt;  // nbr[i * max_nbr + k]

  void build(const double* xyz, int32_t n, double L, double rcs, const Excl& ex, int32_t maxn) {
    max_nbr = maxn;
    nx = std::max(1, (int)(L / rcs));
    const int32_t ncell = nx * nx * nx;
    const bool dedup = nx < 3;
    const double cell = L / nx, inv_cell = 1.0 / cell, inv_L = 1.0 / L;
    const double rcs2 = rcs * rcs;
    std::vector<int32_t> cid(n);
    for (int32_t i = 0; i < n; ++i) {
      int c[3];
      for (int d = 0; d < 3; ++d) {
        int v = (int)std::floor(xyz[3 * i + d] * inv_cell);
        c[d] = ((v % nx) + nx) % nx;
      }
      cid[i] = (c[2] * nx + c[1]) * nx + c[0];
    }
    // Stable sort of atoms by cell id (cub::DeviceRadixSort keeps input order).
    std::vector<int32_t> sorted(n);
    std::iota(sorted.begin(), sorted.end(), 0);
    std::stable_sort(sorted.begin(), sorted.end(), [&](int32_t a, int32_t b) { return cid[a] < cid[b]; });
    std::vector<int32_t> start(ncell, 0), end(ncell, 0);
    for (int32_t k = 0; k < n; ++k) {
      int32_t c = cid[sorted[k]];
      if (k == 0 || cid[sorted[k - 1]] != c) start[c] = k;
      if (k == n - 1 || cid[sorted[k + 1]] != c) end[c] = k + 1;
    }
    nbr.assign((size_t)n * max_nbr, -1);
    cnt.assign(n, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t i = 0; i < n; ++i) {
      const int32_t c = cid[i];
      const int cz = c / (nx * nx), cy = (c / nx) % nx, cx = c % nx;
      int visited[27];
      int nvis = 0;
      int32_t count = 0;
      for (int dz = -1; dz <= 1; ++dz) {
        int ncz = cz + dz;
        if (ncz < 0) ncz += nx; else if (ncz >= nx) ncz -= nx;
        for (int dy = -1; dy <= 1; ++dy) {
          int ncy = cy + dy;
          if (ncy < 0) ncy += nx; else if (ncy >= nx) ncy -= nx;
          for (int dx = -1; dx <= 1; ++dx) {
            int ncx = cx + dx;
            if (ncx < 0) ncx += nx; else if (ncx >= nx) ncx -= nx;
            const int nc = (ncz * nx + ncy) * nx + ncx;
            if (dedup) {
              bool seen = false;
              for (int v = 0; v < nvis; ++v) seen |= (visited[v] == nc);
              if (seen) continue;
              visited[nvis++] = nc;
            }
            for (int32_t b = start[nc]; b < end[nc]; ++b) {
              const int32_t j = sorted[b];
              if (j == i) continue;
              double ddx = min_image(xyz[3 * i] - xyz[3 * j], L, inv_L);
              double ddy = min_image(xyz[3 * i + 1] - xyz[3 * j + 1], L, inv_L);
              double ddz = min_image(xyz[3 * i + 2] - xyz[3 * j + 2], L, inv_L);
              double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
              if (r2 < rcs2 && !ex.has(i, j)) {
                if (count < max_nbr) nbr[(size_t)i * max_nbr + count] = j;
                ++count;
              }
            }
          }
        }
      }
      cnt[i] = count;
    }
  }
};

// ---------------------------------------------------------------------------
// Forces
// ---------------------------------------------------------------------------
struct BondedIndex {
  // atom -> list of (term index, role) for deterministic per-atom gathering
  std::vector<int32_t> b_off, b_item, a_off, a_item;
  void build(const orc_system& s) {
    const int32_t n = s.natoms;
    b_off.assign(n + 1, 0);
    a_off.assign(n + 1, 0);
    for (int32_t b = 0; b < s.nbonds; ++b) {
      b_off[s.bonds[2 * b] + 1]++;
      b_off[s.bonds[2 * b + 1] + 1]++;
    }
    for (int32_t a = 0; a < s.nangles; ++a)
      for (int r = 0; r < 3; ++r) a_off[s.angles[3 * a + r] + 1]++;
    for (int32_t i = 0; i < n; ++i) {
      b_off[i + 1] += b_off[i];
      a_off[i + 1] += a_off[i];
    }
    b_item.assign(b_off[n], 0);
    a_item.assign(a_off[n], 0);
    std::vector<int32_t> fb(b_off.begin(), b_off.end() - 1), fa(a_off.begin(), a_off.end() - 1);
    for (int32_t b = 0; b < s.nbonds; ++b) {
      b_item[fb[s.bonds[2 * b]]++] = 2 * b;
      b_item[fb[s.bonds[2 * b + 1]]++] = 2 * b + 1;
    }
    for (int32_t a = 0; a < s.nangles; ++a)
      for (int r = 0; r < 3; ++r) a_item[fa[s.angles[3 * a + r]]++] = 3 * a + r;
  }
};

// LJ over a Verlet list (force/lj.cu:21-65).  f and pe are overwritten.
void lj_from_list(const orc_system& s, const double* xyz, double L, const Verlet& vl, double* f,
                  double* pe, double* vir) {
  const int32_t n = s.natoms;
  const double inv_L = 1.0 / L, rc2 = s.rc * s.rc;
  std::vector<double> pv((size_t)n * 6);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0, pei = 0;
    double v[6] = {0, 0, 0, 0, 0, 0};
    const int32_t ti = s.type[i];
    const int32_t nn = std::min(vl.cnt[i], vl.max_nbr);
    for (int32_t k = 0; k < nn; ++k) {
      const int32_t j = vl.nbr[(size_t)i * vl.max_nbr + k];
      const int32_t tj = s.type[j];
      double dx = min_image(xyz[3 * i] - xyz[3 * j], L, inv_L);
      double dy = min_image(xyz[3 * i + 1] - xyz[3 * j + 1], L, inv_L);
      double dz = min_image(xyz[3 * i + 2] - xyz[3 * j + 2], L, inv_L);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rc2 && r2 > 1e-10) {
        const double eps = s.lj[2 * (ti * s.ntypes + tj)], sig = s.lj[2 * (ti * s.ntypes + tj) + 1];
        double sig2 = sig * sig;
        double r2inv = 1.0 / r2;
        double sr2 = sig2 * r2inv;
        double sr6 = sr2 * sr2 * sr2;
        double sr12 = sr6 * sr6;
        double fr = 24.0 * eps * r2inv * (2.0 * sr12 - sr6);
        if (s.lj_clamp) fr = std::fmin(std::fmax(fr, -1000.0), 1000.0);
        double fxij = fr * dx, fyij = fr * dy, fzij = fr * dz;
        fx += fxij;
        fy += fyij;
        fz += fzij;
        pei += 0.5 * 4.0 * eps * (sr12 - sr6);
        v[0] += 0.5 * fxij * dx;
        v[1] += 0.5 * fxij * dy;
        v[2] += 0.5 * fxij * dz;
        v[3] += 0.5 * fyij * dy;
        v[4] += 0.5 * fyij * dz;
        v[5] += 0.5 * fzij * dz;
      }
    }
    f[3 * i] = fx;
    f[3 * i + 1] = fy;
    f[3 * i + 2] = fz;
    pe[i] = pei;
    for (int c = 0; c < 6; ++c) pv[(size_t)i * 6 + c] = v[c];
  }
  for (int32_t i = 0; i < n; ++i)
    for (int c = 0; c < 6; ++c) vir[c] += pv[(size_t)i * 6 + c];
}

// FENE + WCA per bond (force/fene.cu:18-73); per-bond results gathered per atom.
void fene_add(const orc_system& s, const BondedIndex& bi, const double* xyz, double L, double* f,
              double* pe, double* vir) {
  const int32_t nb = s.nbonds;
  if (nb == 0) return;
  const double inv_L = 1.0 / L;
  std::vector<double> bf((size_t)nb * 3), bpe(nb), bv((size_t)nb * 6);
#pragma omp parallel for schedule(static)
  for (int32_t b = 0; b < nb; ++b) {
    const int32_t i = s.bonds[2 * b], j = s.bonds[2 * b + 1];
    const double* p = s.fene + 4 * s.bond_type[b];
    const double k = p[0], R0 = p[1], eps = p[2], sig = p[3];
    double dx = min_image(xyz[3 * i] - xyz[3 * j], L, inv_L);
    double dy = min_image(xyz[3 * i + 1] - xyz[3 * j + 1], L, inv_L);
    double dz = min_image(xyz[3 * i + 2] - xyz[3 * j + 2], L, inv_L);
    double r2 = dx * dx + dy * dy + dz * dz;
    double R02 = R0 * R0;
    double r2s = s.fene_clamp ? std::fmin(std::fmax(r2, 1e-6), R02 * 0.9999) : r2;
    double fene_ff = -k * R02 / (R02 - r2s);
    double sig2 = sig * sig;
    double r_cut2 = sig2 * 1.2599210498948732;
    double wca_ff = 0.0, wca_pe = 0.0;
    if (r2s < r_cut2) {
      double r2inv = 1.0 / r2s;
      double sr2 = sig2 * r2inv;
      double sr6 = sr2 * sr2 * sr2;
      double sr12 = sr6 * sr6;
      wca_ff = 24.0 * eps * r2inv * (2.0 * sr12 - sr6);
      wca_pe = 4.0 * eps * (sr12 - sr6) + eps;
    }
    double tot = fene_ff + wca_ff;
    double fix = tot * dx, fiy = tot * dy, fiz = tot * dz;
    double fene_pe = -0.5 * k * R02 * std::log(1.0 - r2s / R02);
    bf[3 * b] = fix;
    bf[3 * b + 1] = fiy;
    bf[3 * b + 2] = fiz;
    bpe[b] = fene_pe + wca_pe;
    double* v = &bv[(size_t)b * 6];
    v[0] = fix * dx;
    v[1] = fix * dy;
    v[2] = fix * dz;
    v[3] = fiy * dy;
    v[4] = fiy * dz;
    v[5] = fiz * dz;
  }
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < s.natoms; ++i) {
    for (int32_t e = bi.b_off[i]; e < bi.b_off[i + 1]; ++e) {
      const int32_t item = bi.b_item[e], b = item >> 1;
      const double sg = (item & 1) ? -1.0 : 1.0;
      f[3 * i] += sg * bf[3 * b];
      f[3 * i + 1] += sg * bf[3 * b + 1];
      f[3 * i + 2] += sg * bf[3 * b + 2];
      pe[i] += 0.5 * bpe[b];
    }
  }
  for (int32_t b = 0; b < nb; ++b)
    for (int c = 0; c < 6; ++c) vir[c] += bv[(size_t)b * 6 + c];
}

// Harmonic angle E = k (theta - theta0)^2 (force/angle.cu:17-80).
void angle_add(const orc_system& s, const BondedIndex& bi, const double* xyz, double L, double* f,
               double* pe, double* vir) {
  const int32_t na = s.nangles;
  if (na == 0) return;
  const double inv_L = 1.0 / L;
  std::vector<double> af((size_t)na * 9), ape(na), av((size_t)na * 6);
#pragma omp parallel for schedule(static)
  for (int32_t a = 0; a < na; ++a) {
    const int32_t i = s.angles[3 * a], j = s.angles[3 * a + 1], k = s.angles[3 * a + 2];
    const double kt = s.angle_p[2 * s.angle_type[a]], th0 = s.angle_p[2 * s.angle_type[a] + 1];
    double dxij = min_image(xyz[3 * i] - xyz[3 * j], L, inv_L);
    double dyij = min_image(xyz[3 * i + 1] - xyz[3 * j + 1], L, inv_L);
    double dzij = min_image(xyz[3 * i + 2] - xyz[3 * j + 2], L, inv_L);
    double dxkj = min_image(xyz[3 * k] - xyz[3 * j], L, inv_L);
    double dykj = min_image(xyz[3 * k + 1] - xyz[3 * j + 1], L, inv_L);
    double dzkj = min_image(xyz[3 * k + 2] - xyz[3 * j + 2], L, inv_L);
    double rij2 = dxij * dxij + dyij * dyij + dzij * dzij;
    double rkj2 = dxkj * dxkj + dykj * dykj + dzkj * dzkj;
    double rij_inv = 1.0 / std::sqrt(rij2);
    double rkj_inv = 1.0 / std::sqrt(rkj2);
    double cs = (dxij * dxkj + dyij * dykj + dzij * dzkj) * rij_inv * rkj_inv;
    cs = std::fmin(std::fmax(cs, -1.0), 1.0);
    double theta = std::acos(cs);
    double dth = theta - th0;
    double sn = std::sqrt(1.0 - cs * cs);
    sn = std::fmax(sn, 1e-6);
    double pref = 2.0 * kt * dth / sn;
    double rij2_inv = 1.0 / rij2, rkj2_inv = 1.0 / rkj2, rr = rij_inv * rkj_inv;
    double* o = &af[(size_t)a * 9];
    o[0] = pref * (dxkj * rr - cs * dxij * rij2_inv);
    o[1] = pref * (dykj * rr - cs * dyij * rij2_inv);
    o[2] = pref * (dzkj * rr - cs * dzij * rij2_inv);
    o[6] = pref * (dxij * rr - cs * dxkj * rkj2_inv);
    o[7] = pref * (dyij * rr - cs * dykj * rkj2_inv);
    o[8] = pref * (dzij * rr - cs * dzkj * rkj2_inv);
    o[3] = -(o[0] + o[6]);
    o[4] = -(o[1] + o[7]);
    o[5] = -(o[2] + o[8]);
    ape[a] = kt * dth * dth;
    double* v = &av[(size_t)a * 6];
    v[0] = o[0] * dxij + o[6] * dxkj;
    v[1] = o[0] * dyij + o[6] * dykj;
    v[2] = o[0] * dzij + o[6] * dzkj;
    v[3] = o[1] * dyij + o[7] * dykj;
    v[4] = o[1] * dzij + o[7] * dzkj;
    v[5] = o[2] * dzij + o[8] * dzkj;
  }
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < s.natoms; ++i) {
    for (int32_t e = bi.a_off[i]; e < bi.a_off[i + 1]; ++e) {
      const int32_t item = bi.a_item[e], a = item / 3, r = item % 3;
      f[3 * i] += af[(size_t)a * 9 + 3 * r];
      f[3 * i + 1] += af[(size_t)a * 9 + 3 * r + 1];
      f[3 * i + 2] += af[(size_t)a * 9 + 3 * r + 2];
      pe[i] += ape[a] / 3.0;
    }
  }
  for (int32_t a = 0; a < na; ++a)
    for (int c = 0; c < 6; ++c) vir[c] += av[(size_t)a * 6 + c];
}

int32_t default_max_nbr(int32_t n, double L, double rcs) {
  // neighbor/verlet_list.cu:4-7
  double density = n / (L * L * L);
  double sphere = (4.0 / 3.0) * 3.14159265358979323846 * rcs * rcs * rcs;
  int est = (int)(density * sphere * 3.0);
  return std::max(256, est);
}

void cap_forces(int32_t n, double cap, double* f) {
  if (cap <= 0) return;
  for (int32_t i = 0; i < n; ++i) {
    double m2 = f[3 * i] * f[3 * i] + f[3 * i + 1] * f[3 * i + 1] + f[3 * i + 2] * f[3 * i + 2];
    if (m2 > cap * cap) {
      double sc = cap / std::sqrt(m2);
      f[3 * i] *= sc;
      f[3 * i + 1] *= sc;
      f[3 * i + 2] *= sc;
    }
  }
}

// Nose-Hoover chain half step: host nh_propagate_chain (nose_hoover.cu:356-447)
// with nh_expf (nose_hoover.cu:72-84), here in double precision.
double nh_exp6(double x) {
  double x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x, x6 = x5 * x;
  return 1.0 + x + x2 * 0.5 + x3 * (1.0 / 6.0) + x4 * (1.0 / 24.0) + x5 * (1.0 / 120.0) +
         x6 * (1.0 / 720.0);
}

// dd_keep: NULL for the reference's scheme (every half step starts its
// upper-chain accelerations from zero, nose_hoover.cu:101, :251, :369); otherwise
// they are read from it and stored back, as LAMMPS's fix nh keeps
// eta_dotdot between calls (the run.conf nh_chain_carry option).
void nhc_half(double* xi, double* vxi, int M, double Q1, double Qr, double kT, int natoms,
              double total_KE, double half_dt, double* scale_out, double* dd_keep = nullptr) {
  const double Nf = 3.0 * (double)natoms;
  const double dt2 = half_dt, dt4 = half_dt * 0.5, dt8 = half_dt * 0.25;
  double dd[10] = {0};
  if (dd_keep)
    for (int k = 1; k < 10; ++k) dd[k] = dd_keep[k];
  double T = (2.0 * total_KE) / Nf;
  if (Q1 > 0.0) dd[0] = (Nf * T - Nf * kT) / Q1;
  const double ncfac = 1.0;
  for (int ich = M - 1; ich > 0; --ich) {
    double ef = (ich + 1 < M) ? nh_exp6(-ncfac * dt8 * vxi[ich + 1]) : 1.0;
    vxi[ich] *= ef;
    vxi[ich] += dd[ich] * ncfac * dt4;
    vxi[ich] *= ef;
  }
  double ef0 = (M > 1) ? nh_exp6(-ncfac * dt8 * vxi[1]) : 1.0;
  vxi[0] *= ef0;
  vxi[0] += dd[0] * ncfac * dt4;
  vxi[0] *= ef0;
  double fe = nh_exp6(-ncfac * dt2 * vxi[0]);
  *scale_out = fe;
  T *= fe * fe;
  if (Q1 > 0.0) dd[0] = (Nf * T - Nf * kT) / Q1;
  for (int ich = 0; ich < M; ++ich) xi[ich] += ncfac * dt2 * vxi[ich];
  vxi[0] *= ef0;
  vxi[0] += dd[0] * ncfac * dt4;
  vxi[0] *= ef0;
  for (int ich = 1; ich < M; ++ich) {
    double ef = (ich + 1 < M) ? nh_exp6(-ncfac * dt8 * vxi[ich + 1]) : 1.0;
    vxi[ich] *= ef;
    double Qp = (ich == 1) ? Q1 : Qr;
    dd[ich] = (Qp * vxi[ich - 1] * vxi[ich - 1] - kT) / Qr;
    vxi[ich] += dd[ich] * ncfac * dt4;
    vxi[ich] *= ef;
  }
  if (dd_keep)
    for (int k = 1; k < 10; ++k) dd_keep[k] = dd[k];
}

void set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // namespace

// ===========================================================================
// C interface
// ===========================================================================
extern "C" {

void orc_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  philox10(ctr, k0, k1, out);
}
void orc_normal3(uint64_t seed, uint32_t stream, uint64_t step, uint32_t id, double out[3]) {
  normal3(seed, stream, step, id, out);
}

double orc_min_image(double dr, double L, double inv_L) { return min_image(dr, L, inv_L); }
double orc_wrap(double x, double L, double inv_L) { return x - L * std::floor(x * inv_L); }
float orc_min_image_f32(float dr, float L, float inv_L) { return dr - L * rintf(dr * inv_L); }

// core/morton.cu:4-28 and cpu_reference.hpp:25-39: 10 bits per axis from
// trunc(p * inv_L * 1024) clamped to [0, 1023], interleaved z|y|x.
static uint32_t expand10(uint32_t v) {
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
static uint32_t quant1024(float p, float inv_L) {
  float q = p * inv_L * 1024.0f;
  uint32_t u = (q <= 0.0f) ? 0u : (q >= 4294967040.0f ? 0xFFFFFFFFu : (uint32_t)q);
  return u > 1023u ? 1023u : u;
}
uint32_t orc_morton_key_f32(float x, float y, float z, float inv_L) {
  return (expand10(quant1024(z, inv_L)) << 2) | (expand10(quant1024(y, inv_L)) << 1) |
         expand10(quant1024(x, inv_L));
}
// cpu_reference.hpp:42-53: sort (key, index) pairs ascending.
void orc_morton_sort_f32(const float* xyz, int32_t n, float inv_L, int32_t* perm) {
  std::vector<std::pair<uint32_t, int32_t>> kv(n);
  for (int32_t i = 0; i < n; ++i) kv[i] = {orc_morton_key_f32(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], inv_L), i};
  std::sort(kv.begin(), kv.end());
  for (int32_t i = 0; i < n; ++i) perm[i] = kv[i].second;
}

int64_t orc_pairs_brute(const double* xyz, int32_t n, double L, double rcs, const int32_t* bonds,
                        int32_t nbonds, int32_t* pi, int32_t* pj, int64_t cap) {
  Excl ex;
  ex.build(n, bonds, nbonds);
  const double inv_L = 1.0 / L, rcs2 = rcs * rcs;
  int64_t np = 0;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = i + 1; j < n; ++j) {
      double dx = min_image(xyz[3 * i] - xyz[3 * j], L, inv_L);
      double dy = min_image(xyz[3 * i + 1] - xyz[3 * j + 1], L, inv_L);
      double dz = min_image(xyz[3 * i + 2] - xyz[3 * j + 2], L, inv_L);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rcs2 && !ex.has(i, j)) {
        if (np < cap) {
          pi[np] = i;
          pj[np] = j;
        }
        ++np;
      }
    }
  return np;
}

// The reference's FP32 predicate (cpu_reference.hpp:11-18 with rc+skin, as
// verlet_list.cu:196-201): float min image with rintf, r2 < rcs*rcs in float.
int64_t orc_pairs_brute_f32(const float* xyz, int32_t n, float L, float rcs, const int32_t* bonds,
                            int32_t nbonds, int32_t* pi, int32_t* pj, int64_t cap) {
  Excl ex;
  ex.build(n, bonds, nbonds);
  const float inv_L = 1.0f / L, rcs2 = rcs * rcs;
  int64_t np = 0;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = i + 1; j < n; ++j) {
      float dx = orc_min_image_f32(xyz[3 * i] - xyz[3 * j], L, inv_L);
      float dy = orc_min_image_f32(xyz[3 * i + 1] - xyz[3 * j + 1], L, inv_L);
      float dz = orc_min_image_f32(xyz[3 * i + 2] - xyz[3 * j + 2], L, inv_L);
      float r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rcs2 && !ex.has(i, j)) {
        if (np < cap) {
          pi[np] = i;
          pj[np] = j;
        }
        ++np;
      }
    }
  return np;
}

// Tile list of 32-atom tiles (neighbor/tile_list.cu:5-171), FP32, statement
// order of the reference with every operation rounded on its own (no
// contraction): per tile the axis-aligned box of its positions (padding slots
// beyond natoms contribute +1e30 to the minimum and -1e30 to the maximum),
// then for every ordered tile pair the distance between the boxes' surfaces
// with the minimum image of the centre offset (tile_list.cu:63-99); pairs
// closer than rc_skin listed per tile a in increasing b (CSR).  Returns the
// pair count; at most cap neighbors are written.
int64_t orc_tile_list_aabb(const float* pos4, int32_t natoms, float L, float rc_skin, int32_t* offsets,
                           int32_t* neighbors, int64_t cap) {
  const int32_t T = (natoms + 31) / 32;
  const float inv_L = 1.0f / L;
  std::vector<float> mn(3 * (size_t)T), mx(3 * (size_t)T);
  for (int32_t t = 0; t < T; ++t)
    for (int d = 0; d < 3; ++d) {
      float lo = 1e30f, hi = -1e30f;
      for (int32_t a = t * 32; a < t * 32 + 32; ++a) {
        const float v = a < natoms ? pos4[4 * (size_t)a + d] : 1e30f;
        lo = std::min(lo, v);
        if (a < natoms) hi = std::max(hi, v);
      }
      mn[3 * t + d] = lo;
      mx[3 * t + d] = hi;
    }
  const float rc2 = rc_skin * rc_skin;
  int64_t np = 0;
  for (int32_t a = 0; a < T; ++a) {
    offsets[a] = (int32_t)np;
    for (int32_t b = 0; b < T; ++b) {
      float s2 = 0.0f;
      for (int d = 0; d < 3; ++d) {
        const float ca = 0.5f * (mn[3 * a + d] + mx[3 * a + d]), cb = 0.5f * (mn[3 * b + d] + mx[3 * b + d]);
        const float ea = 0.5f * (mx[3 * a + d] - mn[3 * a + d]), eb = 0.5f * (mx[3 * b + d] - mn[3 * b + d]);
        float g = std::fabs(orc_min_image_f32(ca - cb, L, inv_L)) - ea - eb;
        g = std::max(g, 0.0f);
        s2 = s2 + g * g;
      }
      if (s2 < rc2) {
        if (np < cap) neighbors[np] = b;
        ++np;
      }
    }
  }
  offsets[T] = (int32_t)np;
  return np;
}

int32_t orc_verlet_lists(const double* xyz, int32_t n, double L, double rcs, const int32_t* bonds,
                         int32_t nbonds, int32_t max_nbr, int32_t* nbr, int32_t* counts) {
  Excl ex;
  ex.build(n, bonds, nbonds);
  Verlet vl;
  vl.build(xyz, n, L, rcs, ex, max_nbr);
  std::memcpy(nbr, vl.nbr.data(), sizeof(int32_t) * (size_t)n * max_nbr);
  std::memcpy(counts, vl.cnt.data(), sizeof(int32_t) * n);
  return vl.nx;
}

void orc_lj(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir) {
  Excl ex;
  ex.build(sys->natoms, sys->bonds, sys->nbonds);
  Verlet vl;
  const double rcs = sys->rc + sys->skin;
  vl.build(xyz, sys->natoms, L, rcs, ex, default_max_nbr(sys->natoms, L, rcs));
  for (int c = 0; c < 6; ++c) vir[c] = 0;
  lj_from_list(*sys, xyz, L, vl, f, pe, vir);
}
void orc_fene(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir) {
  BondedIndex bi;
  bi.build(*sys);
  std::memset(f, 0, sizeof(double) * 3 * sys->natoms);
  std::memset(pe, 0, sizeof(double) * sys->natoms);
  for (int c = 0; c < 6; ++c) vir[c] = 0;
  fene_add(*sys, bi, xyz, L, f, pe, vir);
}
void orc_angle(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir) {
  BondedIndex bi;
  bi.build(*sys);
  std::memset(f, 0, sizeof(double) * 3 * sys->natoms);
  std::memset(pe, 0, sizeof(double) * sys->natoms);
  for (int c = 0; c < 6; ++c) vir[c] = 0;
  angle_add(*sys, bi, xyz, L, f, pe, vir);
}

int32_t orc_forces(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir) {
  Excl ex;
  ex.build(sys->natoms, sys->bonds, sys->nbonds);
  BondedIndex bi;
  bi.build(*sys);
  Verlet vl;
  const double rcs = sys->rc + sys->skin;
  vl.build(xyz, sys->natoms, L, rcs, ex, default_max_nbr(sys->natoms, L, rcs));
  for (int c = 0; c < 6; ++c) vir[c] = 0;
  lj_from_list(*sys, xyz, L, vl, f, pe, vir);
  fene_add(*sys, bi, xyz, L, f, pe, vir);
  angle_add(*sys, bi, xyz, L, f, pe, vir);
  int32_t over = 0;
  for (int32_t i = 0; i < sys->natoms; ++i) over |= (vl.cnt[i] > vl.max_nbr);
  return over;
}

void orc_nhc_half(double* xi, double* v_xi, int32_t M, double Q1, double Q_rest, double kT,
                  int32_t natoms, double total_KE, double half_dt, double* scale_out) {
  nhc_half(xi, v_xi, M, Q1, Q_rest, kT, natoms, total_KE, half_dt, scale_out);
}

// analysis/thermo.cu:88-117 (KE tensor), :119-138 (PE), :173-189 (row).
void orc_thermo(const double* vel, const int32_t* type, const double* mass, const double* pe,
                const double* vir, int32_t n, double L, double* out) {
  double k[6] = {0, 0, 0, 0, 0, 0}, pes = 0;
  for (int32_t i = 0; i < n; ++i) {
    const double m = mass[type[i]];
    const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
    k[0] += m * vx * vx;
    k[1] += m * vx * vy;
    k[2] += m * vx * vz;
    k[3] += m * vy * vy;
    k[4] += m * vy * vz;
    k[5] += m * vz * vz;
    pes += pe[i];
  }
  const double ke = 0.5 * (k[0] + k[3] + k[5]);
  out[0] = ke / n;
  out[1] = pes / n;
  out[2] = 2.0 * out[0] / 3.0;
  const double V = L * L * L;
  for (int c = 0; c < 6; ++c) out[3 + c] = (k[c] + vir[c]) / V;
}

// analysis/rg.cu:3-69 with main.cu:188-296's grouping of atoms by mol id.
double orc_rg(const double* xyz, const int32_t* image, const int32_t* mol, int32_t n, double L) {
  std::vector<int32_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return mol[a] < mol[b]; });
  double sum = 0;
  int32_t nch = 0;
  for (int32_t s = 0; s < n;) {
    int32_t e = s;
    while (e < n && mol[order[e]] == mol[order[s]]) ++e;
    const int32_t len = e - s;
    double com[3] = {0, 0, 0};
    for (int32_t t = s; t < e; ++t)
      for (int d = 0; d < 3; ++d) com[d] += xyz[3 * order[t] + d] + image[3 * order[t] + d] * L;
    for (int d = 0; d < 3; ++d) com[d] /= len;
    double rg2 = 0;
    for (int32_t t = s; t < e; ++t)
      for (int d = 0; d < 3; ++d) {
        double u = xyz[3 * order[t] + d] + image[3 * order[t] + d] * L - com[d];
        rg2 += u * u;
      }
    sum += std::sqrt(rg2 / len);
    ++nch;
    s = e;
  }
  return nch ? sum / nch : 0.0;
}

// ---------------------------------------------------------------------------
// Whole-step simulation (main.cu:403-736)
// ---------------------------------------------------------------------------
struct orc_sim {
  orc_system sys;
  orc_run run;
  std::vector<int32_t> type, mol, bonds, btype, angles, atype;
  std::vector<double> mass, lj, fene, angp;
  Excl ex;
  BondedIndex bi;
  Verlet vl;
  std::vector<double> x, v, f, pe, xref;
  std::vector<int32_t> img;
  double vir[6];
  double L, V0, Q1, Qr, W;
  double xi[10], vxi[10], eps, veps, carry, nh_scale;
  double dd[10] = {0};  // carried chain accelerations (run.chain_carry)
  // Work of the kinetic barostat term the reference's NPT equations leave out
  // (Martyna-Tuckerman-Klein: d v_eps / dt gains (3 / N_f) 2 KE): with the
  // particle velocities scaled by exp(-(1 + 3 / N_f) v_eps / W dt / 2) but
  // no such term in the barostat force, the extended energy changes at
  // -(3 / N_f) (v_eps / W) 2 KE; this sums that rate over the steps taken,
  // for diagnostics only (orc_sim_conserved_mtk).
  double mtk_work = 0.0;
  int64_t step;
  int64_t rebuilds;
  int32_t since;
  int32_t max_nbr;

  void rebuild() {
    vl.build(x.data(), sys.natoms, L, sys.rc + sys.skin, ex, max_nbr);
    xref = x;
    ++rebuilds;
  }
  void forces() {
    for (int c = 0; c < 6; ++c) vir[c] = 0;
    lj_from_list(sys, x.data(), L, vl, f.data(), pe.data(), vir);
    // Push-off caps the non-bonded (LJ) force only, so bonds stay intact.
    cap_forces(sys.natoms, run.force_cap, f.data());
    fene_add(sys, bi, x.data(), L, f.data(), pe.data(), vir);
    angle_add(sys, bi, x.data(), L, f.data(), pe.data(), vir);
  }
  double ke_raw() const {  // sum m v^2 (nose_hoover.cu:904-939)
    double s = 0;
    for (int32_t i = 0; i < sys.natoms; ++i) {
      const double m = mass[type[i]];
      s += m * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    }
    return s;
  }
  // PBC wrap with image flags (langevin.cu:77-88) and the displacement test
  // against the reference positions (skin_trigger.cuh:6-16); returns max dr^2.
  double wrap_and_disp() {
    const double inv_L = 1.0 / L;
    double mx = 0;
    for (int32_t i = 0; i < sys.natoms; ++i) {
      double d2 = 0;
      for (int d = 0; d < 3; ++d) {
        double r = x[3 * i + d];
        int ix = (int)std::floor(r * inv_L);
        r -= ix * L;
        x[3 * i + d] = r;
        img[3 * i + d] += ix;
        double u = round_image(r - xref[3 * i + d], L, inv_L);
        d2 += u * u;
      }
      mx = std::max(mx, d2);
    }
    return mx;
  }
  double ramp(double a, double b) const {
    double frac = (double)(step - 1) / (double)run.nsteps;
    return a + (b - a) * frac;
  }
  void one_step() {
    ++step;
    const int32_t n = sys.natoms;
    const double dt = run.dt, hdt = 0.5 * dt;
    double maxd2 = 0;
    if (run.ensemble == ORC_LANGEVIN) {
      // integrate/langevin.cu:34-94 with langevin.cu:15-21 coefficients.
      const double kT = ramp(run.T_start, run.T_stop);
      const double gamma = 1.0 / run.Tdamp;
      const double c1 = std::exp(-gamma * dt);
      const double c2 = std::sqrt(1.0 - c1 * c1);
#pragma omp parallel for schedule(static)
      for (int32_t i = 0; i < n; ++i) {
        const double m = mass[type[i]];
        const double hm = hdt / m;
        double xi3[3];
        normal3(run.seed, kStreamLangevin, (uint64_t)step, (uint32_t)i, xi3);
        const double ns = c2 * std::sqrt(kT / m);
        for (int d = 0; d < 3; ++d) {
          double vv = v[3 * i + d] + hm * f[3 * i + d];
          double r = x[3 * i + d] + hdt * vv;
          vv = c1 * vv + ns * xi3[d];
          r = r + hdt * vv;
          v[3 * i + d] = vv;
          x[3 * i + d] = r;
        }
      }
      maxd2 = wrap_and_disp();
    } else if (run.ensemble == ORC_NVT_NH) {
      // main.cu:452-481 -> nose_hoover.cu:86-178 (carry) and :606-664.
      const double kT = ramp(run.T_start, run.T_stop);
      double sc;
      nhc_half(xi, vxi, run.chain_length, Q1, Qr, kT, n, carry, hdt, &sc, run.chain_carry ? dd : nullptr);
      nh_scale = sc;
      for (int32_t i = 0; i < n; ++i) {
        const double hm = hdt / mass[type[i]];
        for (int d = 0; d < 3; ++d) {
          double vv = v[3 * i + d] * sc;
          vv = vv + hm * f[3 * i + d];
          x[3 * i + d] = x[3 * i + d] + dt * vv;
          v[3 * i + d] = vv;
        }
      }
      maxd2 = wrap_and_disp();
    } else {
      // NPT pre-force: main.cu:430-468 -> nose_hoover.cu:185-305 (use_carry) and :683-757.
      const double kT = ramp(run.T_start, run.T_stop);
      const double Nf = 3.0 * n, Nf_inv = 1.0 / Nf;
      double V = V0 * std::exp(3.0 * eps);
      L = std::cbrt(V);
      const double vW = veps / W;
      const double bscale = std::exp(-(1.0 + 3.0 * Nf_inv) * vW * hdt);
      double KE = carry * bscale * bscale;
      const double exp_vW = std::exp(vW * dt);
      const double vWdt = vW * dt;
      double sc;
      nhc_half(xi, vxi, run.chain_length, Q1, Qr, kT, n, KE, hdt, &sc, run.chain_carry ? dd : nullptr);
      nh_scale = sc;
      const double hx = 0.5 * vWdt;
      const double sinhc = (std::fabs(hx) < 1e-6) ? 1.0 + hx * hx / 6.0 : std::sinh(hx) / hx;
      const double fpos = dt * std::exp(hx) * sinhc;
      const double scale = sc * bscale;
      for (int32_t i = 0; i < n; ++i) {
        const double hm = hdt / mass[type[i]];
        for (int d = 0; d < 3; ++d) {
          double vv = v[3 * i + d] * scale;
          vv = vv + hm * f[3 * i + d];
          x[3 * i + d] = x[3 * i + d] * exp_vW + vv * fpos;
          xref[3 * i + d] = xref[3 * i + d] * exp_vW;
          v[3 * i + d] = vv;
        }
      }
      maxd2 = wrap_and_disp();
    }
    // Rebuild policy (main.cu:486-528): skin/2 trigger or every 20 steps.
    ++since;
    const bool trig = maxd2 > (0.5 * sys.skin) * (0.5 * sys.skin);
    if (trig || since >= run.max_steps_between_rebuilds) {
      since = 0;
      rebuild();
    }
    forces();
    if (run.ensemble == ORC_LANGEVIN) {
      // integrate/langevin.cu:109-130
      for (int32_t i = 0; i < n; ++i) {
        const double hm = hdt / mass[type[i]];
        for (int d = 0; d < 3; ++d) v[3 * i + d] = v[3 * i + d] + hm * f[3 * i + d];
      }
    } else if (run.ensemble == ORC_NVT_NH) {
      // main.cu:614-627: v-half + KE (nose_hoover.cu:843-889), chain, scale.
      const double kT = ramp(run.T_start, run.T_stop);
      for (int32_t i = 0; i < n; ++i) {
        const double hm = hdt / mass[type[i]];
        for (int d = 0; d < 3; ++d) v[3 * i + d] = v[3 * i + d] + hm * f[3 * i + d];
      }
      const double KE = ke_raw() * 0.5;
      double sc;
      nhc_half(xi, vxi, run.chain_length, Q1, Qr, kT, n, KE, hdt, &sc, run.chain_carry ? dd : nullptr);
      nh_scale = sc;
      carry = KE * sc * sc;
      for (int32_t i = 0; i < 3 * n; ++i) v[i] *= sc;
    } else {
      // main.cu:580-613: v-half, KE + virial trace, SY barostat + chain, rescale.
      const double kT = ramp(run.T_start, run.T_stop);
      const double Pt = ramp(run.P_start, run.P_stop);
      for (int32_t i = 0; i < n; ++i) {
        const double hm = hdt / mass[type[i]];
        for (int d = 0; d < 3; ++d) v[3 * i + d] = v[3 * i + d] + hm * f[3 * i + d];
      }
      const double Nf = 3.0 * n, Nf_inv = 1.0 / Nf;
      const double total_KE = ke_raw() * 0.5;
      const double vtr = vir[0] + vir[3] + vir[5];
      double V = V0 * std::exp(3.0 * eps);
      const double Pinst = (2.0 * total_KE + vtr) / (3.0 * V);
      const double c = std::cbrt(2.0);
      const double w3[3] = {1.0 / (2.0 - c), -c / (2.0 - c), 1.0 / (2.0 - c)};
      for (int sy = 0; sy < 3; ++sy) {
        const double w = w3[sy] * dt;
        double dv = 3.0 * V * (Pinst - Pt) * w;
        const double vh = veps + 0.5 * dv;
        eps += vh * w / W;
        dv = 3.0 * V0 * std::exp(3.0 * eps) * (Pinst - Pt) * w;
        veps += dv;
      }
      V = V0 * std::exp(3.0 * eps);
      L = std::cbrt(V);
      const double vW = veps / W;
      mtk_work += 3.0 * Nf_inv * vW * dt * 2.0 * total_KE;
      const double bscale = std::exp(-(1.0 + 3.0 * Nf_inv) * vW * hdt);
      double KE = total_KE * bscale * bscale;
      double sc;
      nhc_half(xi, vxi, run.chain_length, Q1, Qr, kT, n, KE, hdt, &sc, run.chain_carry ? dd : nullptr);
      nh_scale = sc;
      carry = KE * sc * sc;
      for (int32_t i = 0; i < 3 * n; ++i) v[i] = (v[i] * bscale) * sc;
    }
  }
};


orc_sim* orc_sim_create(const orc_system* sys, const orc_run* run, double L, const double* xyz,
                        const double* vel, const int32_t* image) {
  orc_sim* s = new orc_sim();
  const int32_t n = sys->natoms;
  s->type.assign(sys->type, sys->type + n);
  if (sys->mol) s->mol.assign(sys->mol, sys->mol + n);
  else s->mol.assign(n, 1);
  s->mass.assign(sys->mass, sys->mass + sys->ntypes);
  s->lj.assign(sys->lj, sys->lj + 2 * sys->ntypes * sys->ntypes);
  s->bonds.assign(sys->bonds, sys->bonds + 2 * sys->nbonds);
  s->btype.assign(sys->bond_type, sys->bond_type + sys->nbonds);
  s->fene.assign(sys->fene, sys->fene + 4 * std::max(sys->nbond_types, 0));
  s->angles.assign(sys->angles, sys->angles + 3 * sys->nangles);
  s->atype.assign(sys->angle_type, sys->angle_type + sys->nangles);
  s->angp.assign(sys->angle_p, sys->angle_p + 2 * std::max(sys->nangle_types, 0));
  s->sys = *sys;
  s->sys.type = s->type.data();
  s->sys.mol = s->mol.data();
  s->sys.mass = s->mass.data();
  s->sys.lj = s->lj.data();
  s->sys.bonds = s->bonds.data();
  s->sys.bond_type = s->btype.data();
  s->sys.fene = s->fene.data();
  s->sys.angles = s->angles.data();
  s->sys.angle_type = s->atype.data();
  s->sys.angle_p = s->angp.data();
  s->run = *run;
  if (s->run.max_steps_between_rebuilds <= 0) s->run.max_steps_between_rebuilds = 20;
  set_threads(run->nthreads);
  s->ex.build(n, s->bonds.data(), sys->nbonds);
  s->bi.build(s->sys);
  s->x.assign(xyz, xyz + 3 * n);
  s->v.assign(vel, vel + 3 * n);
  s->img.assign(3 * n, 0);
  if (image) s->img.assign(image, image + 3 * n);
  s->f.assign(3 * n, 0.0);
  s->pe.assign(n, 0.0);
  s->L = L;
  s->V0 = L * L * L;
  s->step = 0;
  s->rebuilds = 0;
  s->since = 0;
  const double rcs = sys->rc + sys->skin;
  s->max_nbr = default_max_nbr(n, L, rcs) * 2;
  // NoseHooverState::init (nose_hoover.cu:309-346)
  const double Nf = 3.0 * n, kT = run->T_start;
  s->Q1 = Nf * kT * run->Tdamp * run->Tdamp;
  s->Qr = kT * run->Tdamp * run->Tdamp;
  s->W = (Nf + 3.0) * kT * run->Pdamp * run->Pdamp;
  for (int k = 0; k < 10; ++k) s->xi[k] = s->vxi[k] = 0;
  s->eps = s->veps = 0;
  s->nh_scale = 1.0;
  // Setup (main.cu:313-342, 364-390): reference positions, list, first forces,
  // initial chain carry = KE.
  s->rebuild();
  s->rebuilds = 0;
  s->forces();
  s->carry = s->ke_raw() * 0.5;
  return s;
}

int32_t orc_sim_step(orc_sim* s, int64_t nsteps) {
  for (int64_t k = 0; k < nsteps; ++k) s->one_step();
  int32_t over = 0;
  for (int32_t i = 0; i < s->sys.natoms; ++i) over |= (s->vl.cnt[i] > s->vl.max_nbr);
  return over;
}

void orc_sim_get(const orc_sim* s, double* xyz, double* vel, int32_t* image, double* f, double* pe,
                 double* vir) {
  const int32_t n = s->sys.natoms;
  // Positions are reported wrapped into the current box (after an NPT step the
  // barostat has already changed L; the stored positions are still wrapped in
  // the box of the last pre-force update).
  for (int32_t k = 0; k < 3 * n; ++k) {
    double x = s->x[k];
    int32_t im = s->img[k];
    const double fl = std::floor(x / s->L);
    x -= fl * s->L;
    im += (int32_t)fl;
    if (xyz) xyz[k] = x;
    if (image) image[k] = im;
  }
  if (vel) std::memcpy(vel, s->v.data(), sizeof(double) * 3 * n);
  if (f) std::memcpy(f, s->f.data(), sizeof(double) * 3 * n);
  if (pe) std::memcpy(pe, s->pe.data(), sizeof(double) * n);
  if (vir) std::memcpy(vir, s->vir, sizeof(double) * 6);
}

void orc_sim_scalars(const orc_sim* s, double* o) {
  o[0] = s->L;
  o[1] = (double)s->step;
  o[2] = (double)s->rebuilds;
  for (int k = 0; k < 10; ++k) {
    o[3 + k] = s->xi[k];
    o[13 + k] = s->vxi[k];
  }
  o[23] = s->eps;
  o[24] = s->veps;
  o[25] = s->carry;
  o[26] = s->nh_scale;
}

void orc_sim_thermo(const orc_sim* s, double* out9) {
  orc_thermo(s->v.data(), s->type.data(), s->mass.data(), s->pe.data(), s->vir, s->sys.natoms, s->L, out9);
}

double orc_sim_rg(const orc_sim* s) {
  return orc_rg(s->x.data(), s->img.data(), s->mol.data(), s->sys.natoms, s->L);
}

// tests/test_nose_hoover.cu:19-40 (NVT); NPT adds v_eps^2 / (2 W) + P V.
double orc_sim_conserved(const orc_sim* s) {
  const int32_t n = s->sys.natoms;
  const double ke = s->ke_raw() * 0.5;
  double pe = 0;
  for (int32_t i = 0; i < n; ++i) pe += s->pe[i];
  double e = ke + pe;
  if (s->run.ensemble != ORC_LANGEVIN) {
    const double Nf = 3.0 * n, kT = s->ramp(s->run.T_start, s->run.T_stop);
    e += 0.5 * s->Q1 * s->vxi[0] * s->vxi[0] + Nf * kT * s->xi[0];
    for (int k = 1; k < s->run.chain_length; ++k) e += 0.5 * s->Qr * s->vxi[k] * s->vxi[k] + kT * s->xi[k];
  }
  if (s->run.ensemble == ORC_NPT_NH) {
    const double Pt = s->ramp(s->run.P_start, s->run.P_stop);
    e += s->veps * s->veps / (2.0 * s->W) + Pt * s->L * s->L * s->L;
  }
  return e;
}

// The NPT extended energy plus the summed work of the missing kinetic
// barostat term: constant to the integrator's order if that term is the
// only gap between the equations of motion and the extended energy.
double orc_sim_conserved_mtk(const orc_sim* s) { return orc_sim_conserved(s) + s->mtk_work; }

void orc_sim_destroy(orc_sim* s) { delete s; }

}  // extern "C"
