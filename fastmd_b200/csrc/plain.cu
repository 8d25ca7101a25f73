// FP64 plain form: the reference's kernels and step loop, restated in double
// precision for one system.  This is the parity anchor against the FP64 CPU
// oracle and the denominator of the batched form's speed-up, so it keeps the
// reference's structure on purpose:
//   - per-atom full Verlet list in the transposed layout neighbors[k*N + i]
//     built from a cell list with cell edge >= rc + skin (verlet_list.cu:3-376);
//   - thread-per-atom LJ (lj.cu:4-107), thread-per-bond FENE and
//     thread-per-angle kernels with atomic scatter (fene.cu:4-101, angle.cu:4-108);
//   - host-side rebuild test every step (skin_trigger.cuh:18-33, main.cu:484-528).
// Differences from the reference: FP64 throughout; the Philox noise of
// counter_rng.h instead of cuRAND state; neighbor overflow and FENE
// over-stretch are reported instead of silently truncated / clamped; the cell
// grid is re-derived from the current box at each rebuild.
//
// This file is compiled with -fmad=false so every product and sum rounds as
// written, like the oracle (built with -ffp-contract=off).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "counter_rng.h"
#include "dev_common.cuh"
#include "engine.h"
#include "nhc.h"

namespace fmd {
namespace plain {

constexpr int kBlock = 256;

struct Params {
  int n;
  int ntypes;
  double L, inv_L;
  const double* mass;  // [ntypes]
};

__device__ __forceinline__ double min_image(double dr, double L, double inv_L) {
  return dr - L * rint(dr * inv_L);
}

__device__ __forceinline__ int type_of(double4 p) { return (int)p.w; }

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// PBC wrap with image flags (langevin.cu:77-88) and the displacement against
// the reference positions (skin_trigger.cuh:6-16).
__device__ __forceinline__ void wrap_disp(double3& r, int i, int* image, const double4* ref,
                                          unsigned long long* maxdr2, double L, double inv_L) {
  const int ix = (int)floor(r.x * inv_L);
  const int iy = (int)floor(r.y * inv_L);
  const int iz = (int)floor(r.z * inv_L);
  r.x = r.x - ix * L;
  r.y = r.y - iy * L;
  r.z = r.z - iz * L;
  if (image) {
    image[3 * i] += ix;
    image[3 * i + 1] += iy;
    image[3 * i + 2] += iz;
  }
  const double4 q = ref[i];
  double u = r.x - q.x;
  u = u - L * round(u * inv_L);
  double d2 = 0.0 + u * u;
  u = r.y - q.y;
  u = u - L * round(u * inv_L);
  d2 = d2 + u * u;
  u = r.z - q.z;
  u = u - L * round(u * inv_L);
  d2 = d2 + u * u;
  atomic_max_nonneg(maxdr2, d2);
}

// BAOAB B-A-O-A + wrap + displacement (langevin.cu:34-94).
__global__ void k_langevin_pre(double4* pos, double4* vel, const double4* force, const double4* ref,
                               unsigned long long* maxdr2, int* image, Params P, double hdt, double c1,
                               double c2, double kT, uint64_t seed, uint32_t stream, uint64_t step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  double4 r = pos[i];
  double4 v = vel[i];
  const double4 f = force[i];
  const double m = P.mass[type_of(r)];
  const double hm = hdt / m;
  double xi0, xi1, xi2;
  rng_normal3(seed, stream, step, (uint32_t)i, &xi0, &xi1, &xi2);
  const double ns = c2 * sqrt(kT / m);
  double3 rr;
  double vv;
  vv = v.x + hm * f.x;
  rr.x = r.x + hdt * vv;
  vv = c1 * vv + ns * xi0;
  rr.x = rr.x + hdt * vv;
  v.x = vv;
  vv = v.y + hm * f.y;
  rr.y = r.y + hdt * vv;
  vv = c1 * vv + ns * xi1;
  rr.y = rr.y + hdt * vv;
  v.y = vv;
  vv = v.z + hm * f.z;
  rr.z = r.z + hdt * vv;
  vv = c1 * vv + ns * xi2;
  rr.z = rr.z + hdt * vv;
  v.z = vv;
  wrap_disp(rr, i, image, ref, maxdr2, P.L, P.inv_L);
  pos[i] = make_double4(rr.x, rr.y, rr.z, r.w);
  vel[i] = v;
}

// Velocity half kick (langevin.cu:109-130, nose_hoover.cu:506-527).
__global__ void k_kick(double4* vel, const double4* force, const double4* pos, Params P, double hdt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  double4 v = vel[i];
  const double4 f = force[i];
  const double hm = hdt / P.mass[type_of(pos[i])];
  v.x = v.x + hm * f.x;
  v.y = v.y + hm * f.y;
  v.z = v.z + hm * f.z;
  vel[i] = v;
}

// Kick + sum m v^2 (nose_hoover.cu:843-889) when kick != 0, else the sum only
// (:780-825 / :904-939); also the virial trace.
__global__ void k_kick_ke(double4* vel, const double4* force, const double4* pos, Params P, double hdt,
                          int kick, double* ke_out) {
  __shared__ double sm[kBlock / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v2 = 0.0;
  if (i < P.n) {
    double4 v = vel[i];
    const double m = P.mass[type_of(pos[i])];
    if (kick) {
      const double4 f = force[i];
      const double hm = hdt / m;
      v.x = v.x + hm * f.x;
      v.y = v.y + hm * f.y;
      v.z = v.z + hm * f.z;
      vel[i] = v;
    }
    v2 = m * (v.x * v.x + v.y * v.y + v.z * v.z);
  }
  v2 = warp_sum(v2);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v2;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kBlock / 32 ? sm[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) atomicAdd(ke_out, t);
  }
}

__global__ void k_scale_vel(double4* vel, const NHScalars* st, int n, int use_bscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = use_bscale ? st->bscale : st->scale;
  double4 v = vel[i];
  v.x = v.x * s;
  v.y = v.y * s;
  v.z = v.z * s;
  vel[i] = v;
}

// NVT pre-force fused (nose_hoover.cu:606-664).
__global__ void k_nvt_pre(double4* pos, double4* vel, const double4* force, const double4* ref,
                          unsigned long long* maxdr2, int* image, const NHScalars* st, Params P, double hdt,
                          double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const double sc = st->scale;
  const double4 r = pos[i];
  double4 v = vel[i];
  const double4 f = force[i];
  const double hm = hdt / P.mass[type_of(r)];
  double3 rr;
  v.x = v.x * sc;
  v.y = v.y * sc;
  v.z = v.z * sc;
  v.x = v.x + hm * f.x;
  v.y = v.y + hm * f.y;
  v.z = v.z + hm * f.z;
  rr.x = r.x + dt * v.x;
  rr.y = r.y + dt * v.y;
  rr.z = r.z + dt * v.z;
  wrap_disp(rr, i, image, ref, maxdr2, P.L, P.inv_L);
  pos[i] = make_double4(rr.x, rr.y, rr.z, r.w);
  vel[i] = v;
}

// NPT pre-force fused (nose_hoover.cu:683-757); L, inv_L are the new box.
__global__ void k_npt_pre(double4* pos, double4* vel, const double4* force, double4* ref,
                          unsigned long long* maxdr2, int* image, const NHScalars* st, Params P, double hdt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const double sc = st->scale * st->bscale;
  const double ev = st->exp_vW, fp = st->fpos;
  const double4 r = pos[i];
  double4 v = vel[i];
  const double4 f = force[i];
  double4 q = ref[i];
  const double hm = hdt / P.mass[type_of(r)];
  v.x = v.x * sc;
  v.y = v.y * sc;
  v.z = v.z * sc;
  v.x = v.x + hm * f.x;
  v.y = v.y + hm * f.y;
  v.z = v.z + hm * f.z;
  double3 rr;
  rr.x = r.x * ev + v.x * fp;
  rr.y = r.y * ev + v.y * fp;
  rr.z = r.z * ev + v.z * fp;
  q.x = q.x * ev;
  q.y = q.y * ev;
  q.z = q.z * ev;
  ref[i] = q;
  wrap_disp(rr, i, image, ref, maxdr2, P.L, P.inv_L);
  pos[i] = make_double4(rr.x, rr.y, rr.z, r.w);
  vel[i] = v;
}

__global__ void k_nvt_chain(NHScalars* st, const double* ke_raw, int pre_force, int M, double Q1, double Qr,
                            double kT, double hdt, int natoms) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double ke = pre_force ? st->carry : (*ke_raw) * 0.5;
  const double sc = nhc_half_step(st->xi, st->vxi, M, Q1, Qr, kT, natoms, ke, hdt, st->carry_dd ? st->dd : nullptr);
  st->scale = sc;
  if (!pre_force) st->carry = ke * sc * sc;
}

struct DevExp {
  __device__ double operator()(double x) const { return exp(x); }
};
struct DevCbrt {
  __device__ double operator()(double x) const { return cbrt(x); }
};
struct DevSinh {
  __device__ double operator()(double x) const { return sinh(x); }
};

__global__ void k_npt_chain(NHScalars* st, const double* ke_raw, const double* virial, int pre_force, int M,
                            double Q1, double Qr, double W, double hdt, double dt, double V0, int natoms,
                            double kT, double Pt) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double vtr = virial[0] + virial[3] + virial[5];
  npt_chain_baro(*st, pre_force != 0, pre_force ? 0.0 : *ke_raw, vtr, M, Q1, Qr, W, hdt, dt, V0, natoms, kT, Pt,
                 DevExp(), DevCbrt(), DevSinh());
}

// ---------------------------------------------------------------- Verlet
// verlet_list.cu:58-75
__global__ void k_assign_cells(const double4* pos, int* cid, int* aid, int n, double inv_cell, int nx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 r = pos[i];
  int cx = (int)floor(r.x * inv_cell), cy = (int)floor(r.y * inv_cell), cz = (int)floor(r.z * inv_cell);
  cx = ((cx % nx) + nx) % nx;
  cy = ((cy % nx) + nx) % nx;
  cz = ((cz % nx) + nx) % nx;
  cid[i] = (cz * nx + cy) * nx + cx;
  aid[i] = i;
}

// verlet_list.cu:82-104
__global__ void k_cell_ranges(const int* scid, int* start, int* end, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = scid[k];
  if (k == 0 || scid[k - 1] != c) start[c] = k;
  if (k == n - 1 || scid[k + 1] != c) end[c] = k + 1;
}

// One thread per atom in cell-sorted order; per atom the candidate order is
// the reference's (27 cells in dz, dy, dx order; cell members in sorted order).
__global__ void k_verlet(const double4* pos, const int* sorted, const int* scid, const int* start, const int* end,
                         const int* eoff, const int* elist, int* nbr, int* cnt, int n, int nx, double rcs2, double L,
                         double inv_L, int max_nbr, int* status) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = sorted[k];
  const int c = scid[k];
  const int cz = c / (nx * nx), cy = (c / nx) % nx, cx = c % nx;
  const bool dedup = nx < 3;
  const double4 pi = pos[i];
  int visited[27];
  int nvis = 0, count = 0;
  const int e0 = eoff ? eoff[i] : 0, e1 = eoff ? eoff[i + 1] : 0;
  for (int dz = -1; dz <= 1; ++dz) {
    int ncz = cz + dz;
    ncz = ncz < 0 ? ncz + nx : (ncz >= nx ? ncz - nx : ncz);
    for (int dy = -1; dy <= 1; ++dy) {
      int ncy = cy + dy;
      ncy = ncy < 0 ? ncy + nx : (ncy >= nx ? ncy - nx : ncy);
      for (int dx = -1; dx <= 1; ++dx) {
        int ncx = cx + dx;
        ncx = ncx < 0 ? ncx + nx : (ncx >= nx ? ncx - nx : ncx);
        const int nc = (ncz * nx + ncy) * nx + ncx;
        if (dedup) {
          bool seen = false;
          for (int v = 0; v < nvis; ++v) seen |= (visited[v] == nc);
          if (seen) continue;
          visited[nvis++] = nc;
        }
        const int b1 = end[nc];
        for (int b = start[nc]; b < b1; ++b) {
          const int j = sorted[b];
          if (j == i) continue;
          const double4 pj = pos[j];
          const double ddx = min_image(pi.x - pj.x, L, inv_L);
          const double ddy = min_image(pi.y - pj.y, L, inv_L);
          const double ddz = min_image(pi.z - pj.z, L, inv_L);
          const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
          if (r2 < rcs2) {
            bool ex = false;
            for (int e = e0; e < e1; ++e) ex |= (elist[e] == j);
            if (!ex) {
              if (count < max_nbr) nbr[(size_t)count * n + i] = j;
              ++count;
            }
          }
        }
      }
    }
  }
  cnt[i] = count < max_nbr ? count : max_nbr;
  if (count > max_nbr) atomicOr(status, kStatusOverflow);
}

// ---------------------------------------------------------------- forces
__device__ __forceinline__ void block_add_virial(double v[6], double* virial) {
  __shared__ double sm[kBlock / 32][6];
  for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 6; ++c) sm[threadIdx.x >> 5][c] = v[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += sm[w][threadIdx.x];
    atomicAdd(&virial[threadIdx.x], s);
  }
}

// lj.cu:4-107 in FP64: force[i] overwritten with (F, pe_i).
__global__ void k_lj(const double4* pos, double4* force, double* virial, const double2* lj, const int* nbr,
                     const int* cnt, int n, int ntypes, double rc2, double L, double inv_L, int clamp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double4 pi = pos[i];
    const int ti = type_of(pi);
    const int nn = cnt[i];
    for (int k = 0; k < nn; ++k) {
      const int j = nbr[(size_t)k * n + i];
      const double4 pj = pos[j];
      const double dx = min_image(pi.x - pj.x, L, inv_L);
      const double dy = min_image(pi.y - pj.y, L, inv_L);
      const double dz = min_image(pi.z - pj.z, L, inv_L);
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rc2 && r2 > 1e-10) {
        const double2 p = lj[ti * ntypes + type_of(pj)];
        const double eps = p.x, sig = p.y;
        const double sig2 = sig * sig;
        const double r2inv = 1.0 / r2;
        const double sr2 = sig2 * r2inv;
        const double sr6 = sr2 * sr2 * sr2;
        const double sr12 = sr6 * sr6;
        double fr = 24.0 * eps * r2inv * (2.0 * sr12 - sr6);
        if (clamp) fr = fmin(fmax(fr, -1000.0), 1000.0);
        const double fxij = fr * dx, fyij = fr * dy, fzij = fr * dz;
        fx += fxij;
        fy += fyij;
        fz += fzij;
        pe += 0.5 * 4.0 * eps * (sr12 - sr6);
        v[0] += 0.5 * fxij * dx;
        v[1] += 0.5 * fxij * dy;
        v[2] += 0.5 * fxij * dz;
        v[3] += 0.5 * fyij * dy;
        v[4] += 0.5 * fyij * dz;
        v[5] += 0.5 * fzij * dz;
      }
    }
    force[i] = make_double4(fx, fy, fz, pe);
  }
  block_add_virial(v, virial);
}

// fene.cu:4-101 in FP64 with atomic scatter; over-stretch reported.
__global__ void k_fene(const double4* pos, double4* force, double* virial, const int2* bonds, const int* btype,
                       const double4* fp, int nb, double L, double inv_L, int clamp, int* status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (b < nb) {
    const int2 bd = bonds[b];
    const double4 p = fp[btype[b]];
    const double k = p.x, R0 = p.y, eps = p.z, sig = p.w;
    const double4 ri = pos[bd.x], rj = pos[bd.y];
    const double dx = min_image(ri.x - rj.x, L, inv_L);
    const double dy = min_image(ri.y - rj.y, L, inv_L);
    const double dz = min_image(ri.z - rj.z, L, inv_L);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double R02 = R0 * R0;
    if (r2 >= R02 * 0.9999) atomicOr(status, kStatusFeneStretch);
    const double r2s = clamp ? fmin(fmax(r2, 1e-6), R02 * 0.9999) : r2;
    const double fene_ff = -k * R02 / (R02 - r2s);
    const double sig2 = sig * sig;
    const double rcut2 = sig2 * 1.2599210498948732;
    double wff = 0.0, wpe = 0.0;
    if (r2s < rcut2) {
      const double r2inv = 1.0 / r2s;
      const double sr2 = sig2 * r2inv;
      const double sr6 = sr2 * sr2 * sr2;
      const double sr12 = sr6 * sr6;
      wff = 24.0 * eps * r2inv * (2.0 * sr12 - sr6);
      wpe = 4.0 * eps * (sr12 - sr6) + eps;
    }
    const double tot = fene_ff + wff;
    const double fix = tot * dx, fiy = tot * dy, fiz = tot * dz;
    atomicAdd(&force[bd.x].x, fix);
    atomicAdd(&force[bd.x].y, fiy);
    atomicAdd(&force[bd.x].z, fiz);
    atomicAdd(&force[bd.y].x, -fix);
    atomicAdd(&force[bd.y].y, -fiy);
    atomicAdd(&force[bd.y].z, -fiz);
    const double fpe = -0.5 * k * R02 * log(1.0 - r2s / R02);
    const double ppe = fpe + wpe;
    atomicAdd(&force[bd.x].w, 0.5 * ppe);
    atomicAdd(&force[bd.y].w, 0.5 * ppe);
    v[0] = fix * dx;
    v[1] = fix * dy;
    v[2] = fix * dz;
    v[3] = fiy * dy;
    v[4] = fiy * dz;
    v[5] = fiz * dz;
  }
  block_add_virial(v, virial);
}

// angle.cu:4-108 in FP64 with atomic scatter.
__global__ void k_angle(const double4* pos, double4* force, double* virial, const int4* angles, const double2* ap,
                        int na, double L, double inv_L) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (a < na) {
    const int4 an = angles[a];
    const double2 p = ap[an.w];
    const double kt = p.x, th0 = p.y;
    const double4 ri = pos[an.x], rj = pos[an.y], rk = pos[an.z];
    const double dxij = min_image(ri.x - rj.x, L, inv_L);
    const double dyij = min_image(ri.y - rj.y, L, inv_L);
    const double dzij = min_image(ri.z - rj.z, L, inv_L);
    const double dxkj = min_image(rk.x - rj.x, L, inv_L);
    const double dykj = min_image(rk.y - rj.y, L, inv_L);
    const double dzkj = min_image(rk.z - rj.z, L, inv_L);
    const double rij2 = dxij * dxij + dyij * dyij + dzij * dzij;
    const double rkj2 = dxkj * dxkj + dykj * dykj + dzkj * dzkj;
    const double rij_inv = 1.0 / sqrt(rij2);
    const double rkj_inv = 1.0 / sqrt(rkj2);
    double cs = (dxij * dxkj + dyij * dykj + dzij * dzkj) * rij_inv * rkj_inv;
    cs = fmin(fmax(cs, -1.0), 1.0);
    const double theta = acos(cs);
    const double dth = theta - th0;
    double sn = sqrt(1.0 - cs * cs);
    sn = fmax(sn, 1e-6);
    const double pref = 2.0 * kt * dth / sn;
    const double rij2_inv = 1.0 / rij2, rkj2_inv = 1.0 / rkj2, rr = rij_inv * rkj_inv;
    const double fix = pref * (dxkj * rr - cs * dxij * rij2_inv);
    const double fiy = pref * (dykj * rr - cs * dyij * rij2_inv);
    const double fiz = pref * (dzkj * rr - cs * dzij * rij2_inv);
    const double fkx = pref * (dxij * rr - cs * dxkj * rkj2_inv);
    const double fky = pref * (dyij * rr - cs * dykj * rkj2_inv);
    const double fkz = pref * (dzij * rr - cs * dzkj * rkj2_inv);
    atomicAdd(&force[an.x].x, fix);
    atomicAdd(&force[an.x].y, fiy);
    atomicAdd(&force[an.x].z, fiz);
    atomicAdd(&force[an.z].x, fkx);
    atomicAdd(&force[an.z].y, fky);
    atomicAdd(&force[an.z].z, fkz);
    atomicAdd(&force[an.y].x, -(fix + fkx));
    atomicAdd(&force[an.y].y, -(fiy + fky));
    atomicAdd(&force[an.y].z, -(fiz + fkz));
    const double pe = kt * dth * dth;
    const double third = pe / 3.0;
    atomicAdd(&force[an.x].w, third);
    atomicAdd(&force[an.y].w, third);
    atomicAdd(&force[an.z].w, third);
    v[0] = fix * dxij + fkx * dxkj;
    v[1] = fix * dyij + fkx * dykj;
    v[2] = fix * dzij + fkx * dzkj;
    v[3] = fiy * dyij + fky * dykj;
    v[4] = fiy * dzij + fky * dzkj;
    v[5] = fiz * dzij + fkz * dzkj;
  }
  block_add_virial(v, virial);
}

__global__ void k_cap(double4* force, int n, double cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 f = force[i];
  const double m2 = f.x * f.x + f.y * f.y + f.z * f.z;
  if (m2 > cap * cap) {
    const double s = cap / sqrt(m2);
    f.x *= s;
    f.y *= s;
    f.z *= s;
    force[i] = f;
  }
}

// thermo.cu:88-138: KE tensor and PE sum (out[0..5], out[6]); non-finite check.
__global__ void k_thermo(const double4* vel, const double4* pos, const double4* force, Params P, double* out,
                         int* status) {
  __shared__ double sm[kBlock / 32][7];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  if (i < P.n) {
    const double4 v = vel[i];
    const double4 r = pos[i];
    const double m = P.mass[type_of(r)];
    s[0] = m * v.x * v.x;
    s[1] = m * v.x * v.y;
    s[2] = m * v.x * v.z;
    s[3] = m * v.y * v.y;
    s[4] = m * v.y * v.z;
    s[5] = m * v.z * v.z;
    s[6] = force[i].w;
    if (!isfinite(s[0] + s[3] + s[5] + s[6] + r.x + r.y + r.z)) atomicOr(status, kStatusNonFinite);
  }
  for (int c = 0; c < 7; ++c) s[c] = warp_sum(s[c]);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 7; ++c) sm[threadIdx.x >> 5][c] = s[c];
  __syncthreads();
  if (threadIdx.x < 7) {
    double t = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) t += sm[w][threadIdx.x];
    atomicAdd(&out[threadIdx.x], t);
  }
}

// rg.cu:3-69: one block per chain, atoms of the chain listed in order[off..].
__global__ void k_rg(const double4* pos, const int* image, const int* order, const int* off, double L,
                     double* sum) {
  __shared__ double sm[3][kBlock / 32];
  const int c = blockIdx.x;
  const int s = off[c], e = off[c + 1], len = e - s;
  double cx = 0, cy = 0, cz = 0;
  for (int t = s + threadIdx.x; t < e; t += blockDim.x) {
    const int i = order[t];
    const double4 r = pos[i];
    cx += r.x + image[3 * i] * L;
    cy += r.y + image[3 * i + 1] * L;
    cz += r.z + image[3 * i + 2] * L;
  }
  cx = warp_sum(cx);
  cy = warp_sum(cy);
  cz = warp_sum(cz);
  if ((threadIdx.x & 31) == 0) {
    sm[0][threadIdx.x >> 5] = cx;
    sm[1][threadIdx.x >> 5] = cy;
    sm[2][threadIdx.x >> 5] = cz;
  }
  __syncthreads();
  double com[3] = {0, 0, 0};
  for (int w = 0; w < kBlock / 32; ++w)
    for (int d = 0; d < 3; ++d) com[d] += sm[d][w];
  for (int d = 0; d < 3; ++d) com[d] /= len;
  __syncthreads();
  double rg2 = 0;
  for (int t = s + threadIdx.x; t < e; t += blockDim.x) {
    const int i = order[t];
    const double4 r = pos[i];
    const double ux = r.x + image[3 * i] * L - com[0];
    const double uy = r.y + image[3 * i + 1] * L - com[1];
    const double uz = r.z + image[3 * i + 2] * L - com[2];
    rg2 += ux * ux + uy * uy + uz * uz;
  }
  rg2 = warp_sum(rg2);
  if ((threadIdx.x & 31) == 0) sm[0][threadIdx.x >> 5] = rg2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < kBlock / 32; ++w) t += sm[0][w];
    atomicAdd(sum, sqrt(t / len));
  }
}

// ---------------------------------------------------------------- engine
class PlainEngine final : public SimEngine {
 public:
  PlainEngine(const RunConfig& cfg, Topology topo, const fmd_melt_spec* pushoff) : cfg_(cfg), t_(std::move(topo)) {
    n_ = t_.natoms;
    L_ = t_.box_L;
    V0_ = L_ * L_ * L_;
    const int32_t nt = cfg_.ntypes;
    FMD_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    // state
    std::vector<double4> h(n_);
    for (int i = 0; i < n_; ++i) h[i] = make_double4(t_.xyz[3 * i], t_.xyz[3 * i + 1], t_.xyz[3 * i + 2], (double)t_.type[i]);
    pos_.alloc(n_);
    FMD_CUDA(cudaMemcpy(pos_, h.data(), n_ * sizeof(double4), cudaMemcpyHostToDevice));
    for (int i = 0; i < n_; ++i) h[i] = make_double4(t_.vel[3 * i], t_.vel[3 * i + 1], t_.vel[3 * i + 2], 0.0);
    vel_.alloc(n_);
    FMD_CUDA(cudaMemcpy(vel_, h.data(), n_ * sizeof(double4), cudaMemcpyHostToDevice));
    force_.alloc_zero(n_);
    ref_.alloc(n_);
    image_.alloc(3 * (size_t)n_);
    FMD_CUDA(cudaMemcpy(image_, t_.image.data(), 3 * n_ * sizeof(int), cudaMemcpyHostToDevice));
    mass_.alloc(nt);
    FMD_CUDA(cudaMemcpy(mass_, t_.mass.data(), nt * sizeof(double), cudaMemcpyHostToDevice));
    lj_.alloc((size_t)nt * nt);
    FMD_CUDA(cudaMemcpy(lj_, cfg_.lj.data(), (size_t)nt * nt * sizeof(double2), cudaMemcpyHostToDevice));
    // topology
    nb_ = t_.nbonds();
    na_ = t_.nangles();
    if (nb_) {
      bonds_.alloc(nb_);
      FMD_CUDA(cudaMemcpy(bonds_, t_.bonds.data(), nb_ * sizeof(int2), cudaMemcpyHostToDevice));
      btype_.alloc(nb_);
      FMD_CUDA(cudaMemcpy(btype_, t_.bond_type.data(), nb_ * sizeof(int), cudaMemcpyHostToDevice));
      std::vector<double4> fp(cfg_.bond.size());
      for (size_t k = 0; k < fp.size(); ++k) fp[k] = make_double4(cfg_.bond[k][0], cfg_.bond[k][1], cfg_.bond[k][2], cfg_.bond[k][3]);
      fene_.alloc(fp.size());
      FMD_CUDA(cudaMemcpy(fene_, fp.data(), fp.size() * sizeof(double4), cudaMemcpyHostToDevice));
      std::vector<int32_t> eo, el;
      build_exclusions(t_, eo, el);
      eoff_.alloc(eo.size());
      FMD_CUDA(cudaMemcpy(eoff_, eo.data(), eo.size() * sizeof(int), cudaMemcpyHostToDevice));
      elist_.alloc(std::max<size_t>(1, el.size()));
      if (!el.empty()) FMD_CUDA(cudaMemcpy(elist_, el.data(), el.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (na_) {
      std::vector<int4> a(na_);
      for (int k = 0; k < na_; ++k) a[k] = make_int4(t_.angles[3 * k], t_.angles[3 * k + 1], t_.angles[3 * k + 2], t_.angle_type[k]);
      angles_.alloc(na_);
      FMD_CUDA(cudaMemcpy(angles_, a.data(), na_ * sizeof(int4), cudaMemcpyHostToDevice));
      std::vector<double2> ap(cfg_.angle.size());
      for (size_t k = 0; k < ap.size(); ++k) ap[k] = make_double2(cfg_.angle[k][0], cfg_.angle[k][1]);
      angp_.alloc(ap.size());
      FMD_CUDA(cudaMemcpy(angp_, ap.data(), ap.size() * sizeof(double2), cudaMemcpyHostToDevice));
    }
    // Verlet storage: the grid is sized for a box up to 1.5x the initial edge.
    rcs_ = cfg_.rc + cfg_.skin;
    max_nbr_ = reference_max_neighbors(n_, L_, rcs_);
    const int nx_max = std::max(1, (int)(1.5 * L_ / rcs_));
    cell_cap_ = nx_max * nx_max * nx_max;
    nbr_.alloc((size_t)max_nbr_ * n_);
    cnt_.alloc_zero(n_);
    cid_.alloc(n_);
    scid_.alloc(n_);
    aid_.alloc(n_);
    sorted_.alloc(n_);
    cstart_.alloc(cell_cap_);
    cend_.alloc(cell_cap_);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr, n_);
    cub_tmp_.alloc(tb);
    maxdr2_.alloc_zero(1);
    virial_.alloc_zero(6);
    status_.alloc_zero(1);
    red_.alloc_zero(8);
    nh_.alloc_zero(1);
    // Rg chains: atoms grouped by mol id (main.cu:188-296 sorts by mol id).
    {
      std::vector<int32_t> order(n_);
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return t_.mol[a] < t_.mol[b]; });
      std::vector<int32_t> off = {0};
      for (int k = 1; k < n_; ++k)
        if (t_.mol[order[k]] != t_.mol[order[k - 1]]) off.push_back(k);
      off.push_back(n_);
      nchains_ = (int)off.size() - 1;
      rg_order_.alloc(n_);
      FMD_CUDA(cudaMemcpy(rg_order_, order.data(), n_ * sizeof(int), cudaMemcpyHostToDevice));
      rg_off_.alloc(off.size());
      FMD_CUDA(cudaMemcpy(rg_off_, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    // Thermostat constants (NoseHooverState::init, nose_hoover.cu:309-346).
    const double Nf = 3.0 * n_, kT0 = cfg_.T_start;
    Q1_ = Nf * kT0 * cfg_.Tdamp * cfg_.Tdamp;
    Qr_ = kT0 * cfg_.Tdamp * cfg_.Tdamp;
    W_ = (Nf + 3.0) * kT0 * cfg_.Pdamp * cfg_.Pdamp;
    {
      NHScalars s;
      std::memset(&s, 0, sizeof(s));
      s.scale = 1.0;
      s.bscale = 1.0;
      s.exp_vW = 1.0;
      s.L = L_;
      s.inv_L = 1.0 / L_;
      s.V = V0_;
      s.carry_dd = cfg_.nh_chain_carry;
      FMD_CUDA(cudaMemcpy(nh_, &s, sizeof(s), cudaMemcpyHostToDevice));
    }
    setup_forces();
    if (pushoff && pushoff->pushoff_steps > 0) run_pushoff(*pushoff);
    init_carry();
  }

  ~PlainEngine() override {
    if (st_) cudaStreamDestroy(st_);
  }

  void step(int64_t nsteps) override {
    for (int64_t k = 0; k < nsteps; ++k) one_step(cfg_.dt, 0.0, kStreamLangevin, cfg_.ensemble);
    sync_check();
  }

  void compute_forces(double* f, double* pe, double* vir) override {
    std::vector<double4> h(n_);
    FMD_CUDA(cudaMemcpyAsync(h.data(), force_, n_ * sizeof(double4), cudaMemcpyDeviceToHost, st_));
    double v[6];
    FMD_CUDA(cudaMemcpyAsync(v, virial_, sizeof(v), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
    for (int i = 0; i < n_; ++i) {
      if (f) {
        f[3 * i] = h[i].x;
        f[3 * i + 1] = h[i].y;
        f[3 * i + 2] = h[i].z;
      }
      if (pe) pe[i] = h[i].w;
    }
    if (vir) std::memcpy(vir, v, sizeof(v));
  }

  void get_state(double* xyz, double* vel, int32_t* image) override {
    std::vector<double4> h(n_);
    std::vector<int32_t> img(3 * n_);
    FMD_CUDA(cudaMemcpy(img.data(), image_, 3 * n_ * sizeof(int), cudaMemcpyDeviceToHost));
    if (xyz || image) {
      // Reported wrapped into the current box (the barostat may have changed
      // L after the last pre-force wrap).
      FMD_CUDA(cudaMemcpy(h.data(), pos_, n_ * sizeof(double4), cudaMemcpyDeviceToHost));
      for (int i = 0; i < n_; ++i) {
        const double r[3] = {h[i].x, h[i].y, h[i].z};
        for (int a = 0; a < 3; ++a) {
          const double fl = std::floor(r[a] / L_);
          if (xyz) xyz[3 * i + a] = r[a] - fl * L_;
          img[3 * i + a] += (int32_t)fl;
        }
      }
    }
    if (vel) {
      FMD_CUDA(cudaMemcpy(h.data(), vel_, n_ * sizeof(double4), cudaMemcpyDeviceToHost));
      for (int i = 0; i < n_; ++i) {
        vel[3 * i] = h[i].x;
        vel[3 * i + 1] = h[i].y;
        vel[3 * i + 2] = h[i].z;
      }
    }
    if (image) std::memcpy(image, img.data(), 3 * n_ * sizeof(int32_t));
  }

  void set_state(const double* xyz, const double* vel, const int32_t* image) override {
    std::vector<double4> h(n_);
    if (xyz) {
      std::vector<int32_t> img(image ? std::vector<int32_t>(image, image + 3 * n_) : std::vector<int32_t>(3 * n_, 0));
      for (int i = 0; i < n_; ++i) {
        double r[3];
        for (int d = 0; d < 3; ++d) {
          r[d] = xyz[3 * i + d];
          const double fl = std::floor(r[d] / L_);
          r[d] -= fl * L_;
          img[3 * i + d] += (int)fl;
          if (r[d] >= L_) { r[d] -= L_; img[3 * i + d] += 1; }
          if (r[d] < 0) r[d] = 0;
        }
        h[i] = make_double4(r[0], r[1], r[2], (double)t_.type[i]);
      }
      FMD_CUDA(cudaMemcpy(pos_, h.data(), n_ * sizeof(double4), cudaMemcpyHostToDevice));
      FMD_CUDA(cudaMemcpy(image_, img.data(), 3 * n_ * sizeof(int), cudaMemcpyHostToDevice));
    } else if (image) {
      FMD_CUDA(cudaMemcpy(image_, image, 3 * n_ * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (vel) {
      for (int i = 0; i < n_; ++i) h[i] = make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 0.0);
      FMD_CUDA(cudaMemcpy(vel_, h.data(), n_ * sizeof(double4), cudaMemcpyHostToDevice));
    }
    setup_forces();
    init_carry();
  }

  void checkpoint(Topology& t, StateFile& s) override {
    t.xyz.resize(3 * (size_t)n_);
    t.vel.resize(3 * (size_t)n_);
    t.image.resize(3 * (size_t)n_);
    get_state(t.xyz.data(), t.vel.data(), t.image.data());
    t.box_L = L_;
    NHScalars nh;
    FMD_CUDA(cudaMemcpy(&nh, nh_, sizeof(nh), cudaMemcpyDeviceToHost));
    s.put("form", {0.0});
    s.put("natoms", {(double)n_});
    s.put("ensemble", {(double)cfg_.ensemble});
    s.put("step", {(double)step_});
    s.put("box_L", {L_});
    s.put("V0", {V0_});
    s.put("rebuilds", {(double)rebuilds_});
    s.put("nh_xi", std::vector<double>(nh.xi, nh.xi + 10));
    s.put("nh_vxi", std::vector<double>(nh.vxi, nh.vxi + 10));
    s.put("nh_scalars", {nh.eps, nh.veps, nh.carry, nh.scale, nh.L, nh.inv_L, nh.V, nh.bscale, nh.exp_vW, nh.vWdt,
                         nh.fpos, nh.ke_raw, nh.vir_tr});
    s.put("nh_dd", std::vector<double>(nh.dd, nh.dd + 10));
    restore(t, s);
  }

  void restore(const Topology& t, const StateFile& s) override {
    if ((int)s.get1("natoms") != n_) throw Error(FMD_ERR_IO, "restart state is for another atom count");
    if ((int)s.get1("ensemble") != cfg_.ensemble) throw Error(FMD_ERR_IO, "restart state is for another ensemble");
    step_ = (int64_t)s.get1("step");
    L_ = s.get1("box_L");
    V0_ = s.get1("V0");
    set_state(t.xyz.data(), t.vel.data(), t.image.data());
    if (s.has("rebuilds")) rebuilds_ = (int64_t)s.get1("rebuilds");
    NHScalars nh;
    FMD_CUDA(cudaMemcpy(&nh, nh_, sizeof(nh), cudaMemcpyDeviceToHost));
    const auto& xi = s.get("nh_xi");
    const auto& vxi = s.get("nh_vxi");
    const auto& c = s.get("nh_scalars");
    if (xi.size() != 10 || vxi.size() != 10 || c.size() != 13) throw Error(FMD_ERR_IO, "bad chain state in sidecar");
    for (int k = 0; k < 10; ++k) {
      nh.xi[k] = xi[k];
      nh.vxi[k] = vxi[k];
    }
    nh.eps = c[0];
    nh.veps = c[1];
    nh.carry = c[2];
    nh.scale = c[3];
    nh.L = c[4];
    nh.inv_L = c[5];
    nh.V = c[6];
    nh.bscale = c[7];
    nh.exp_vW = c[8];
    nh.vWdt = c[9];
    nh.fpos = c[10];
    nh.ke_raw = c[11];
    nh.vir_tr = c[12];
    if (s.has("nh_dd")) {
      const auto& dd = s.get("nh_dd");
      if (dd.size() != 10) throw Error(FMD_ERR_IO, "bad chain state in sidecar");
      for (int k = 0; k < 10; ++k) nh.dd[k] = dd[k];
    }
    FMD_CUDA(cudaMemcpy(nh_, &nh, sizeof(nh), cudaMemcpyHostToDevice));
  }

  void thermo(fmd_thermo_row* row) override {
    FMD_CUDA(cudaMemsetAsync(red_, 0, 8 * sizeof(double), st_));
    k_thermo<<<div_up(n_, kBlock), kBlock, 0, st_>>>(vel_, pos_, force_, params(), red_, status_);
    FMD_CUDA_LAUNCH();
    double s[8], v[6];
    FMD_CUDA(cudaMemcpyAsync(s, red_, sizeof(s), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaMemcpyAsync(v, virial_, sizeof(v), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
    const double ke = 0.5 * (s[0] + s[3] + s[5]);
    row->step = step_;
    row->ke = ke / n_;
    row->pe = s[6] / n_;
    row->temp = 2.0 * row->ke / 3.0;
    const double V = L_ * L_ * L_;
    for (int c = 0; c < 6; ++c) row->stress[c] = (s[c] + v[c]) / V;
    row->box_L = L_;
    row->conserved = conserved(ke, s[6]) / n_;
  }

  double rg() override {
    FMD_CUDA(cudaMemsetAsync(red_, 0, sizeof(double), st_));
    k_rg<<<nchains_, kBlock, 0, st_>>>(pos_, image_, rg_order_, rg_off_, L_, red_);
    FMD_CUDA_LAUNCH();
    double s;
    FMD_CUDA(cudaMemcpyAsync(&s, red_, sizeof(s), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
    return s / nchains_;
  }

  int64_t pairs(int32_t* pi, int32_t* pj, int64_t cap) override {
    std::vector<int32_t> nb((size_t)max_nbr_ * n_), c(n_);
    FMD_CUDA(cudaMemcpy(nb.data(), nbr_, nb.size() * sizeof(int), cudaMemcpyDeviceToHost));
    FMD_CUDA(cudaMemcpy(c.data(), cnt_, n_ * sizeof(int), cudaMemcpyDeviceToHost));
    int64_t m = 0;
    for (int i = 0; i < n_; ++i)
      for (int k = 0; k < c[i]; ++k) {
        const int j = nb[(size_t)k * n_ + i];
        if (j > i) {
          if (m < cap) {
            pi[m] = i;
            pj[m] = j;
          }
          ++m;
        }
      }
    return m;
  }

  int32_t natoms() const override { return n_; }
  int32_t nbonds() const override { return nb_; }
  int32_t nangles() const override { return na_; }
  int64_t step_count() const override { return step_; }
  double box_L() override { return L_; }
  int64_t rebuilds() const override { return rebuilds_; }
  int32_t status_word() override {
    int32_t s = 0;
    FMD_CUDA(cudaMemcpy(&s, status_, sizeof(int), cudaMemcpyDeviceToHost));
    return s;
  }
  int32_t max_neighbors() const override { return max_nbr_; }

 private:
  Params params() const { return Params{n_, cfg_.ntypes, L_, 1.0 / L_, mass_}; }

  double ramp(double a, double b) const {
    const double frac = (double)(step_ - 1) / (double)(cfg_.nsteps > 0 ? cfg_.nsteps : 1);
    return a + (b - a) * frac;
  }

  void rebuild() {
    const int nx = std::max(1, (int)(L_ / rcs_));
    if ((long long)nx * nx * nx > cell_cap_) {
      FMD_CUDA(cudaMemsetAsync(status_, 0, sizeof(int), st_));  // keep the word simple: report below
      throw Error(FMD_ERR_OVERFLOW, "cell grid outgrew its allocation (box expanded beyond 1.5x)");
    }
    const int ncell = nx * nx * nx;
    const double cell = L_ / nx, inv_cell = 1.0 / cell;
    const int g = div_up(n_, kBlock);
    k_assign_cells<<<g, kBlock, 0, st_>>>(pos_, cid_, aid_, n_, inv_cell, nx);
    FMD_CUDA_LAUNCH();
    size_t tb = cub_tmp_.bytes();
    FMD_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tb, cid_.p, scid_.p, aid_.p, sorted_.p, n_, 0, 32, st_));
    FMD_CUDA(cudaMemsetAsync(cstart_, 0, ncell * sizeof(int), st_));
    FMD_CUDA(cudaMemsetAsync(cend_, 0, ncell * sizeof(int), st_));
    k_cell_ranges<<<g, kBlock, 0, st_>>>(scid_, cstart_, cend_, n_);
    FMD_CUDA_LAUNCH();
    k_verlet<<<g, kBlock, 0, st_>>>(pos_, sorted_, scid_, cstart_, cend_, nb_ ? eoff_.p : nullptr,
                                    nb_ ? elist_.p : nullptr, nbr_, cnt_, n_, nx, rcs_ * rcs_, L_, 1.0 / L_,
                                    max_nbr_, status_);
    FMD_CUDA_LAUNCH();
    FMD_CUDA(cudaMemcpyAsync(ref_, pos_, n_ * sizeof(double4), cudaMemcpyDeviceToDevice, st_));
    ++rebuilds_;
  }

  void forces(double cap) {
    FMD_CUDA(cudaMemsetAsync(virial_, 0, 6 * sizeof(double), st_));
    k_lj<<<div_up(n_, kBlock), kBlock, 0, st_>>>(pos_, force_, virial_, lj_, nbr_, cnt_, n_, cfg_.ntypes,
                                                 cfg_.rc * cfg_.rc, L_, 1.0 / L_, 1);
    FMD_CUDA_LAUNCH();
    if (cap > 0) {  // push-off caps the non-bonded force only
      k_cap<<<div_up(n_, kBlock), kBlock, 0, st_>>>(force_, n_, cap);
      FMD_CUDA_LAUNCH();
    }
    if (nb_) {
      k_fene<<<div_up(nb_, kBlock), kBlock, 0, st_>>>(pos_, force_, virial_, bonds_, btype_, fene_, nb_, L_,
                                                      1.0 / L_, 1, status_);
      FMD_CUDA_LAUNCH();
    }
    if (na_) {
      k_angle<<<div_up(na_, kBlock), kBlock, 0, st_>>>(pos_, force_, virial_, angles_, angp_, na_, L_, 1.0 / L_);
      FMD_CUDA_LAUNCH();
    }
  }

  void setup_forces() {
    // main.cu:313-342: reference positions, list, first forces.
    FMD_CUDA(cudaMemsetAsync(maxdr2_, 0, sizeof(unsigned long long), st_));
    rebuild();
    rebuilds_ = 0;
    since_ = 0;
    forces(0.0);
    FMD_CUDA(cudaStreamSynchronize(st_));
  }

  void init_carry() {
    // main.cu:376-390: chain carry starts at the current KE.
    FMD_CUDA(cudaMemsetAsync(red_, 0, sizeof(double), st_));
    k_kick_ke<<<div_up(n_, kBlock), kBlock, 0, st_>>>(vel_, force_, pos_, params(), 0.0, 0, red_);
    FMD_CUDA_LAUNCH();
    double ke;
    FMD_CUDA(cudaMemcpyAsync(&ke, red_, sizeof(double), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
    NHScalars s;
    FMD_CUDA(cudaMemcpy(&s, nh_, sizeof(s), cudaMemcpyDeviceToHost));
    s.carry = 0.5 * ke;
    FMD_CUDA(cudaMemcpy(nh_, &s, sizeof(s), cudaMemcpyHostToDevice));
  }

  void run_pushoff(const fmd_melt_spec& sp) {
    const double dt = sp.pushoff_dt > 0 ? sp.pushoff_dt : 0.005;
    const double cap = sp.pushoff_fcap > 0 ? sp.pushoff_fcap : 50.0;
    forces(cap);
    for (int k = 0; k < sp.pushoff_steps; ++k) one_step(dt, cap, kStreamPushoff, FMD_LANGEVIN);
    sync_check();
    step_ = 0;
    setup_forces();
  }

  double conserved(double ke, double pe) {
    if (cfg_.ensemble == FMD_LANGEVIN) return ke + pe;
    NHScalars s;
    FMD_CUDA(cudaMemcpy(&s, nh_, sizeof(s), cudaMemcpyDeviceToHost));
    const double Nf = 3.0 * n_, kT = ramp(cfg_.T_start, cfg_.T_stop);
    double e = ke + pe + 0.5 * Q1_ * s.vxi[0] * s.vxi[0] + Nf * kT * s.xi[0];
    for (int k = 1; k < cfg_.chain_length; ++k) e += 0.5 * Qr_ * s.vxi[k] * s.vxi[k] + kT * s.xi[k];
    if (cfg_.ensemble == FMD_NPT_NH) e += s.veps * s.veps / (2.0 * W_) + ramp(cfg_.P_start, cfg_.P_stop) * L_ * L_ * L_;
    return e;
  }

  void sync_check() {
    FMD_CUDA(cudaStreamSynchronize(st_));
    const int32_t s = status_word();
    if (s & kStatusOverflow) throw Error(FMD_ERR_OVERFLOW, "neighbor list overflow");
    if (s & (kStatusNonFinite | kStatusFeneStretch))
      throw Error(FMD_ERR_FAULT, (s & kStatusNonFinite) ? "non-finite state" : "FENE bond stretched to R0");
  }

  // main.cu:403-736 for one step.
  void one_step(double dt, double cap, uint32_t stream, int ensemble) {
    ++step_;
    const double hdt = 0.5 * dt;
    const int g = div_up(n_, kBlock);
    const int M = cfg_.chain_length;
    if (ensemble == FMD_LANGEVIN) {
      const double kT = ramp(cfg_.T_start, cfg_.T_stop);
      const double gamma = 1.0 / cfg_.Tdamp;
      const double c1 = std::exp(-gamma * dt);
      const double c2 = std::sqrt(1.0 - c1 * c1);
      k_langevin_pre<<<g, kBlock, 0, st_>>>(pos_, vel_, force_, ref_, maxdr2_, image_, params(), hdt, c1, c2, kT,
                                            cfg_.seed, stream, (uint64_t)step_);
    } else if (ensemble == FMD_NVT_NH) {
      const double kT = ramp(cfg_.T_start, cfg_.T_stop);
      k_nvt_chain<<<1, 1, 0, st_>>>(nh_, nullptr, 1, M, Q1_, Qr_, kT, hdt, n_);
      k_nvt_pre<<<g, kBlock, 0, st_>>>(pos_, vel_, force_, ref_, maxdr2_, image_, nh_, params(), hdt, dt);
    } else {
      const double kT = ramp(cfg_.T_start, cfg_.T_stop), Pt = ramp(cfg_.P_start, cfg_.P_stop);
      k_npt_chain<<<1, 1, 0, st_>>>(nh_, red_, virial_, 1, M, Q1_, Qr_, W_, hdt, dt, V0_, n_, kT, Pt);
      read_box();  // main.cu:453-456
      k_npt_pre<<<g, kBlock, 0, st_>>>(pos_, vel_, force_, ref_, maxdr2_, image_, nh_, params(), hdt);
    }
    FMD_CUDA_LAUNCH();
    // Rebuild test on the host every step (skin_trigger.cuh:18-33, main.cu:484-528).
    ++since_;
    unsigned long long bits = 0;
    FMD_CUDA(cudaMemcpyAsync(&bits, maxdr2_, sizeof(bits), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
    double maxd2;
    std::memcpy(&maxd2, &bits, sizeof(double));
    const double hs = 0.5 * cfg_.skin;
    if (maxd2 > hs * hs || since_ >= 20) {
      FMD_CUDA(cudaMemsetAsync(maxdr2_, 0, sizeof(bits), st_));
      since_ = 0;
      rebuild();
    }
    forces(cap);
    if (ensemble == FMD_LANGEVIN) {
      k_kick<<<g, kBlock, 0, st_>>>(vel_, force_, pos_, params(), hdt);
    } else if (ensemble == FMD_NVT_NH) {
      const double kT = ramp(cfg_.T_start, cfg_.T_stop);
      FMD_CUDA(cudaMemsetAsync(red_, 0, sizeof(double), st_));
      k_kick_ke<<<g, kBlock, 0, st_>>>(vel_, force_, pos_, params(), hdt, 1, red_);
      k_nvt_chain<<<1, 1, 0, st_>>>(nh_, red_, 0, M, Q1_, Qr_, kT, hdt, n_);
      k_scale_vel<<<g, kBlock, 0, st_>>>(vel_, nh_, n_, 0);
    } else {
      const double kT = ramp(cfg_.T_start, cfg_.T_stop), Pt = ramp(cfg_.P_start, cfg_.P_stop);
      FMD_CUDA(cudaMemsetAsync(red_, 0, sizeof(double), st_));
      k_kick_ke<<<g, kBlock, 0, st_>>>(vel_, force_, pos_, params(), hdt, 1, red_);
      k_npt_chain<<<1, 1, 0, st_>>>(nh_, red_, virial_, 0, M, Q1_, Qr_, W_, hdt, dt, V0_, n_, kT, Pt);
      k_scale_vel<<<g, kBlock, 0, st_>>>(vel_, nh_, n_, 1);
      k_scale_vel<<<g, kBlock, 0, st_>>>(vel_, nh_, n_, 0);
      read_box();  // main.cu:610-613
    }
    FMD_CUDA_LAUNCH();
  }

  void read_box() {
    NHScalars s;
    FMD_CUDA(cudaMemcpyAsync(&s, nh_, sizeof(s), cudaMemcpyDeviceToHost, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
    L_ = s.L;
  }

  RunConfig cfg_;
  Topology t_;
  int32_t n_ = 0, nb_ = 0, na_ = 0, nchains_ = 0;
  double L_ = 0, V0_ = 0, rcs_ = 0, Q1_ = 0, Qr_ = 0, W_ = 0;
  int32_t max_nbr_ = 0;
  long long cell_cap_ = 0;
  int64_t step_ = 0, rebuilds_ = 0;
  int32_t since_ = 0;
  cudaStream_t st_ = nullptr;
  DevBuf<double4> pos_, vel_, force_, ref_;
  DevBuf<int> image_;
  DevBuf<double> mass_;
  DevBuf<double2> lj_;
  DevBuf<int2> bonds_;
  DevBuf<int> btype_;
  DevBuf<double4> fene_;
  DevBuf<int4> angles_;
  DevBuf<double2> angp_;
  DevBuf<int> eoff_, elist_;
  DevBuf<int> nbr_, cnt_, cid_, scid_, aid_, sorted_, cstart_, cend_;
  DevBuf<char> cub_tmp_;
  DevBuf<unsigned long long> maxdr2_;
  DevBuf<double> virial_, red_;
  DevBuf<int> status_;
  DevBuf<NHScalars> nh_;
  DevBuf<int> rg_order_, rg_off_;
};

}  // namespace plain

std::unique_ptr<SimEngine> make_plain_engine(const RunConfig& cfg, Topology topo, const fmd_melt_spec* pushoff) {
  if (!cfg.tables.empty()) throw Error(FMD_ERR_CONFIG, "tabulated pair potentials are computed by the mixed form");
  if (cfg.stress_on) throw Error(FMD_ERR_CONFIG, "the stress autocorrelation is computed by the mixed form");
  return std::unique_ptr<SimEngine>(new plain::PlainEngine(cfg, std::move(topo), pushoff));
}

}  // namespace fmd
