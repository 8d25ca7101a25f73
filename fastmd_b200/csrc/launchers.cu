// Reference-layout launchers: drop-in replacements for the reference's
// in-process entry points that take raw device pointers and a stream.
//   fmd_launch_verlet_build  <- VerletList::build   (neighbor/verlet_list.cu:337-376)
//   fmd_launch_lj            <- launch_lj_kernel    (force/lj.cu:109-122)
//   fmd_launch_morton_sort   <- MortonSorter::sort_and_permute (core/morton.cu:65-85)
//   fmd_launch_tile_list     <- TileList::build     (neighbor/tile_list.cu:143-171)
//   fmd_launch_lj_tiles      <- the LJ pass over TileList's pairs (warp per tile)
// Buffers keep the reference's layout: float4 positions with the type id
// bit-cast into .w, the transposed list neighbors[k * natoms + i].
// FP32 throughout, as the reference; this file is compiled with -fmad=false so
// the pair predicate rounds exactly like reference/cpu_reference.hpp on the
// host (the pair set is bit-exact against it).  Differences: neighbor overflow
// raises a flag instead of truncating silently; the caller owns all memory.
#include <cub/cub.cuh>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "dev_common.cuh"
#include "host.h"

namespace fmd {
namespace launch {

constexpr int kBlock = 256;

__device__ __forceinline__ float min_image_f(float dr, float L, float inv_L) { return dr - L * rintf(dr * inv_L); }

struct VerletGeom {
  int nx, ncell;
  float cell, inv_cell;
};

// Cells per axis above which the cubed cell count no longer fits an int
// (1290^3 > 2^31); larger grids are refused before any size is computed.
constexpr int kMaxCellsPerAxis = 1290;

// verlet_list.cu:3-13 (grid from the box) with the same FP32 arithmetic.
// Refuses a box or cutoff that is not finite and positive, and a grid whose
// cell count would overflow (the reference computes nx^3 in int).
inline VerletGeom verlet_geom(float L, float rcs) {
  if (!(std::isfinite(L) && std::isfinite(rcs) && L > 0.0f && rcs > 0.0f))
    throw Error(FMD_ERR_ARG, "box_L and rc_skin must be finite and positive");
  const float per_axis = L / rcs;
  if (!std::isfinite(per_axis) || per_axis >= (float)kMaxCellsPerAxis)
    throw Error(FMD_ERR_CAPACITY, "cell grid too large: box_L / rc_skin must stay below " +
                                      std::to_string(kMaxCellsPerAxis));
  VerletGeom g;
  g.nx = (int)per_axis;
  if (g.nx < 1) g.nx = 1;
  const int64_t ncell = (int64_t)g.nx * g.nx * g.nx;
  g.ncell = (int)ncell;
  g.cell = L / (float)g.nx;
  g.inv_cell = 1.0f / g.cell;
  return g;
}

struct VerletScratch {
  int* cid;
  int* cid_sorted;
  int* aid;
  int* sorted;
  int* start;
  int* end;
  void* cub;
  size_t cub_bytes;
  size_t total;
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

VerletScratch verlet_carve(void* base, int n, int ncell) {
  VerletScratch s{};
  size_t cub_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr, n);
  char* p = (char*)base;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* q = p ? p + off : nullptr;
    off += align256(bytes);
    return q;
  };
  s.cid = (int*)take(sizeof(int) * n);
  s.cid_sorted = (int*)take(sizeof(int) * n);
  s.aid = (int*)take(sizeof(int) * n);
  s.sorted = (int*)take(sizeof(int) * n);
  s.start = (int*)take(sizeof(int) * ncell);
  s.end = (int*)take(sizeof(int) * ncell);
  s.cub = take(cub_bytes);
  s.cub_bytes = cub_bytes;
  s.total = off;
  return s;
}

// verlet_list.cu:58-75
__global__ void k_assign(const float4* pos, int* cid, int* aid, int n, float inv_cell, int nx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r = pos[i];
  int cx = __float2int_rd(r.x * inv_cell), cy = __float2int_rd(r.y * inv_cell), cz = __float2int_rd(r.z * inv_cell);
  cx = ((cx % nx) + nx) % nx;
  cy = ((cy % nx) + nx) % nx;
  cz = ((cz % nx) + nx) % nx;
  cid[i] = (cz * nx + cy) * nx + cx;
  aid[i] = i;
}

__global__ void k_ranges(const int* scid, int* start, int* end, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = scid[k];
  if (k == 0 || scid[k - 1] != c) start[c] = k;
  if (k == n - 1 || scid[k + 1] != c) end[c] = k + 1;
}

// One thread per atom in cell-sorted order; per atom the candidate order is
// the reference's (verlet_list.cu:154-327).
__global__ void k_build(const float4* pos, const int* sorted, const int* scid, const int* start, const int* end,
                        const int* eoff, const int* elist, int* nbr, int* cnt, int n, int nx, float rcs2, float L,
                        float inv_L, int max_nbr, int* overflow) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = sorted[k];
  const int c = scid[k];
  const int cz = c / (nx * nx), cy = (c / nx) % nx, cx = c % nx;
  const bool dedup = nx < 3;
  const float4 pi = pos[i];
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
          const float4 pj = __ldg(&pos[j]);
          const float ddx = min_image_f(pi.x - pj.x, L, inv_L);
          const float ddy = min_image_f(pi.y - pj.y, L, inv_L);
          const float ddz = min_image_f(pi.z - pj.z, L, inv_L);
          const float r2 = ddx * ddx + ddy * ddy + ddz * ddz;
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
  if (count > max_nbr && overflow) atomicOr(overflow, 1);
}

// lj.cu:4-107 semantics: force[i] = (F, pe_i) overwritten, virial accumulated.
// One pair's force on i, half its energy and half its virial (lj.cu:32-61):
// F/r clamped to +-1000 (lj.cu:48).  p = (eps, sigma) of the type pair.
__device__ __forceinline__ void lj_ref_pair(float2 p, float dx, float dy, float dz, float r2, float& fx, float& fy,
                                            float& fz, float& pe, float* v) {
  const float sig2 = p.y * p.y;
  const float r2inv = __fdividef(1.0f, r2);
  const float sr2 = sig2 * r2inv;
  const float sr6 = sr2 * sr2 * sr2;
  const float sr12 = sr6 * sr6;
  float fr = 24.0f * p.x * r2inv * (2.0f * sr12 - sr6);
  fr = fminf(fmaxf(fr, -1000.0f), 1000.0f);
  const float fxij = fr * dx, fyij = fr * dy, fzij = fr * dz;
  fx += fxij;
  fy += fyij;
  fz += fzij;
  pe += 0.5f * 4.0f * p.x * (sr12 - sr6);
  v[0] += 0.5f * fxij * dx;
  v[1] += 0.5f * fxij * dy;
  v[2] += 0.5f * fxij * dz;
  v[3] += 0.5f * fyij * dy;
  v[4] += 0.5f * fyij * dz;
  v[5] += 0.5f * fzij * dz;
}

__global__ void k_lj(const float4* __restrict__ pos, float4* __restrict__ force, float* __restrict__ virial,
                     const float2* __restrict__ lj, const int* __restrict__ nbr, const int* __restrict__ cnt, int n,
                     int ntypes, float rc2, float L, float inv_L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float fx = 0, fy = 0, fz = 0, pe = 0;
  float v[6] = {0, 0, 0, 0, 0, 0};
  if (i < n) {
    const float4 pi = pos[i];
    const int ti = __float_as_int(pi.w);
    const int nn = __ldg(&cnt[i]);
    for (int k = 0; k < nn; ++k) {
      const int j = __ldg(&nbr[(size_t)k * n + i]);
      const float4 pj = __ldg(&pos[j]);
      const float dx = min_image_f(pi.x - pj.x, L, inv_L);
      const float dy = min_image_f(pi.y - pj.y, L, inv_L);
      const float dz = min_image_f(pi.z - pj.z, L, inv_L);
      const float r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rc2 && r2 > 1e-10f)
        lj_ref_pair(__ldg(&lj[ti * ntypes + __float_as_int(pj.w)]), dx, dy, dz, r2, fx, fy, fz, pe, v);
    }
    force[i] = make_float4(fx, fy, fz, pe);
  }
  __shared__ float sm[kBlock / 32][6];
  for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 6; ++c) sm[threadIdx.x >> 5][c] = v[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    float s = 0;
    for (int w = 0; w < kBlock / 32; ++w) s += sm[w][threadIdx.x];
    atomicAdd(&virial[threadIdx.x], s);
  }
}

// morton.cu:4-28: 10 bits per axis from trunc(p * inv_L * 1024) clamped.
__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void k_morton_keys(const float4* pos, uint32_t* keys, int* idx, int n, float inv_L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = pos[i];
  const uint32_t ix = min(max(__float2uint_rz(p.x * inv_L * 1024.0f), 0u), 1023u);
  const uint32_t iy = min(max(__float2uint_rz(p.y * inv_L * 1024.0f), 0u), 1023u);
  const uint32_t iz = min(max(__float2uint_rz(p.z * inv_L * 1024.0f), 0u), 1023u);
  keys[i] = (spread10(iz) << 2) | (spread10(iy) << 1) | spread10(ix);
  idx[i] = i;
}

__global__ void k_gather4(float4* dst, const float4* src, const int* perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[perm[i]];
}

struct MortonScratch {
  uint32_t* keys;
  uint32_t* keys_sorted;
  int* idx;
  float4* tmp;
  void* cub;
  size_t cub_bytes;
  size_t total;
};

MortonScratch morton_carve(void* base, int n) {
  MortonScratch s{};
  size_t cub_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int*)nullptr,
                                  (int*)nullptr, n);
  char* p = (char*)base;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* q = p ? p + off : nullptr;
    off += align256(bytes);
    return q;
  };
  s.keys = (uint32_t*)take(sizeof(uint32_t) * n);
  s.keys_sorted = (uint32_t*)take(sizeof(uint32_t) * n);
  s.idx = (int*)take(sizeof(int) * n);
  s.tmp = (float4*)take(sizeof(float4) * n);
  s.cub = take(cub_bytes);
  s.cub_bytes = cub_bytes;
  s.total = off;
  return s;
}

// ---------------------------------------------------------------------------
// Tile list (neighbor/tile_list.cu:5-171): tile pairs of 32-atom tiles whose
// axis-aligned boxes lie within rc_skin (minimum image between box centres),
// as CSR in increasing partner order.  The reference writes ntiles^2 flags
// and scans them (3.9 GB at 10^6 atoms); here one warp per tile tests 32
// partners per ballot, once to count and once to write, with O(ntiles)
// memory.  The predicate keeps the reference's statement order; this file
// is compiled without contraction, so it is exact against the FP32 oracle.
__global__ void k_tile_bbox(const float4* pos, float4* tmin, float4* tmax, int natoms) {
  const int t = blockIdx.x, lane = threadIdx.x;
  const int a = t * 32 + lane;
  float3 lo = make_float3(1e30f, 1e30f, 1e30f), hi = make_float3(-1e30f, -1e30f, -1e30f);
  if (a < natoms) {
    const float4 r = pos[a];
    lo = hi = make_float3(r.x, r.y, r.z);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = fminf(lo.x, __shfl_down_sync(0xffffffffu, lo.x, o));
    lo.y = fminf(lo.y, __shfl_down_sync(0xffffffffu, lo.y, o));
    lo.z = fminf(lo.z, __shfl_down_sync(0xffffffffu, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_down_sync(0xffffffffu, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_down_sync(0xffffffffu, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_down_sync(0xffffffffu, hi.z, o));
  }
  if (lane == 0) {
    tmin[t] = make_float4(lo.x, lo.y, lo.z, 0.f);
    tmax[t] = make_float4(hi.x, hi.y, hi.z, 0.f);
  }
}

// tile_list.cu:63-99: distance between the two boxes' surfaces below rc_skin.
__device__ __forceinline__ bool tiles_near(float4 amin, float4 amax, float4 bmin, float4 bmax, float L,
                                           float inv_L, float rc2) {
  const float cax = 0.5f * (amin.x + amax.x), cay = 0.5f * (amin.y + amax.y), caz = 0.5f * (amin.z + amax.z);
  const float cbx = 0.5f * (bmin.x + bmax.x), cby = 0.5f * (bmin.y + bmax.y), cbz = 0.5f * (bmin.z + bmax.z);
  const float eax = 0.5f * (amax.x - amin.x), eay = 0.5f * (amax.y - amin.y), eaz = 0.5f * (amax.z - amin.z);
  const float ebx = 0.5f * (bmax.x - bmin.x), eby = 0.5f * (bmax.y - bmin.y), ebz = 0.5f * (bmax.z - bmin.z);
  float dx = fabsf(min_image_f(cax - cbx, L, inv_L)) - eax - ebx;
  float dy = fabsf(min_image_f(cay - cby, L, inv_L)) - eay - eby;
  float dz = fabsf(min_image_f(caz - cbz, L, inv_L)) - eaz - ebz;
  dx = fmaxf(dx, 0.0f);
  dy = fmaxf(dy, 0.0f);
  dz = fmaxf(dz, 0.0f);
  return dx * dx + dy * dy + dz * dz < rc2;
}

// WRITE = false: per-tile pair counts (into cnt, entry ntiles set to 0 for the
// scan); WRITE = true: the partners at off[a], at most cap in all.
template <bool WRITE>
__global__ void k_tile_pairs(const float4* tmin, const float4* tmax, int ntiles, float L, float inv_L, float rc2,
                             int* cnt, const int* off, int* nbr, int cap) {
  const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (!WRITE && blockIdx.x == 0 && threadIdx.x == 0) cnt[ntiles] = 0;
  if (a >= ntiles) return;
  const float4 amin = tmin[a], amax = tmax[a];
  int run = WRITE ? off[a] : 0;
  for (int b0 = 0; b0 < ntiles; b0 += 32) {
    const int b = b0 + lane;
    const bool hit = b < ntiles && tiles_near(amin, amax, tmin[b], tmax[b], L, inv_L, rc2);
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (WRITE && hit) {
      const int at = run + __popc(m & ((1u << lane) - 1u));
      if (at < cap) nbr[at] = b;
    }
    run += __popc(m);
  }
  if (!WRITE && lane == 0) cnt[a] = run;
}

// LJ over the tile list, a warp per i-tile (the tile-pair form of the LJ
// pass over TileList's pairs): one lane per i atom; each partner j-tile's 32
// positions are staged in the warp's shared-memory slice (the next partner's
// loaded ahead into a register) and every lane evaluates its atom against
// all 32.  Masked per tile pair: the atom itself, its excluded partners (the
// exclusion CSR the Verlet build takes; one bit per j slot, set from the
// atom's few partners) and slots past natoms.  Each pair is evaluated from
// both tiles (force on i only, half the energy and virial per side) with
// k_lj's pair arithmetic, so the forces differ from k_lj's by summation
// order only.
constexpr int kTileWarps = 4;
__global__ void __launch_bounds__(32 * kTileWarps) k_lj_tiles(const float4* __restrict__ pos,
                                                               float4* __restrict__ force, float* __restrict__ virial,
                                                               const float2* __restrict__ lj,
                                                               const int* __restrict__ toff,
                                                               const int* __restrict__ tnbr,
                                                               const int* __restrict__ xoff,
                                                               const int* __restrict__ xlist, int n, int ntiles,
                                                               int ntypes, float rc2, float L, float inv_L) {
  __shared__ float4 s_pos[kTileWarps][32];
  __shared__ float sm[kTileWarps][6];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = blockIdx.x * kTileWarps + w;
  float fx = 0, fy = 0, fz = 0, pe = 0;
  float v[6] = {0, 0, 0, 0, 0, 0};
  if (a < ntiles) {  // warp-uniform
    const int i = a * 32 + lane;
    const bool live = i < n;
    const float4 pi = live ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int ti = __float_as_int(pi.w);
    const int x0 = live && xoff ? xoff[i] : 0, x1 = live && xoff ? xoff[i + 1] : 0;
    const int p0 = toff[a], p1 = toff[a + 1];
    float4 nxt = make_float4(0.f, 0.f, 0.f, 0.f);
    if (p0 < p1) {
      const int j = tnbr[p0] * 32 + lane;
      if (j < n) nxt = pos[j];
    }
    for (int p = p0; p < p1; ++p) {
      const int jb = tnbr[p] * 32;
      __syncwarp();  // the previous partner's slice is no longer read
      s_pos[w][lane] = nxt;
      if (p + 1 < p1) {
        const int j = tnbr[p + 1] * 32 + lane;
        nxt = j < n ? pos[j] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      __syncwarp();
      uint32_t skip = n - jb >= 32 ? 0u : ~0u << (n - jb);
      if (jb == a * 32) skip |= 1u << lane;
      for (int e = x0; e < x1; ++e) {
        const int jx = xlist[e] - jb;
        if ((unsigned)jx < 32u) skip |= 1u << jx;
      }
      if (live) {
#pragma unroll 4
        for (int jj = 0; jj < 32; ++jj) {
          const float4 pj = s_pos[w][jj];
          const float dx = min_image_f(pi.x - pj.x, L, inv_L);
          const float dy = min_image_f(pi.y - pj.y, L, inv_L);
          const float dz = min_image_f(pi.z - pj.z, L, inv_L);
          const float r2 = dx * dx + dy * dy + dz * dz;
          if (r2 < rc2 && r2 > 1e-10f && !((skip >> jj) & 1u))
            lj_ref_pair(__ldg(&lj[ti * ntypes + __float_as_int(pj.w)]), dx, dy, dz, r2, fx, fy, fz, pe, v);
        }
      }
    }
    if (live) force[i] = make_float4(fx, fy, fz, pe);
  }
  for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
  if (lane == 0)
    for (int c = 0; c < 6; ++c) sm[w][c] = v[c];
  __syncthreads();
  if (threadIdx.x < 6) {
    float s = 0;
    for (int k = 0; k < kTileWarps; ++k) s += sm[k][threadIdx.x];
    atomicAdd(&virial[threadIdx.x], s);
  }
}

struct TileScratch {
  float4* tmin;
  float4* tmax;
  int* cnt;
  void* cub;
  size_t cub_bytes;
  size_t total;
};

TileScratch tile_carve(void* base, int ntiles) {
  TileScratch s{};
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (int*)nullptr, (int*)nullptr, ntiles + 1);
  char* p = (char*)base;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* q = p ? p + off : nullptr;
    off += align256(bytes);
    return q;
  };
  s.tmin = (float4*)take(sizeof(float4) * ntiles);
  s.tmax = (float4*)take(sizeof(float4) * ntiles);
  s.cnt = (int*)take(sizeof(int) * (ntiles + 1));
  s.cub = take(cub_bytes);
  s.cub_bytes = cub_bytes;
  s.total = off;
  return s;
}

// ---------------------------------------------------------------------------
// Allocation-free Verlet build.  Some callers cannot allocate device memory:
// code running inside another framework's memory pool or a stream-capture
// region, or a host process that must not grow its device footprint after
// start-up.  For them the cell-list scratch of fmd_launch_verlet_build lives in
// this fixed array, which every GPU that loads the library holds until the
// process exits.  Its device address is looked up once per device with
// cudaGetSymbolAddress (the array's name in host code is only a host-side
// stand-in, never a device pointer).
constexpr size_t kStaticScratchBytes = (size_t)8 << 20;  // 8 MiB
constexpr int kStaticMaxAtoms = 1 << 17;                  // 131072 atoms
constexpr int kStaticMaxCells = 1 << 16;                  // 65536 cells
constexpr int kStaticMaxCellsPerAxis = 40;                // 40^3 = 64000 cells
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_verlet_static_scratch[kStaticScratchBytes];

static std::mutex g_static_mu;
static void* g_static_ptr[kMaxDevices] = {};

// Device address of the static scratch for the current device (looked up on
// the first call for that device, with that device current, and kept for the
// life of the process: a cudaDeviceReset on that device invalidates it, and
// calls after such a reset are not supported).
void* static_scratch_for_current_device() {
  int dev = 0;
  FMD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(FMD_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_verlet_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      throw Error(FMD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    g_static_ptr[dev] = p;
  }
  return g_static_ptr[dev];
}

}  // namespace launch
}  // namespace fmd

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
  } catch (const std::exception& e) {
    fmd::set_last_error(e.what());
    return FMD_ERR_ARG;
  }
}
}  // namespace

using namespace fmd;
using namespace fmd::launch;

extern "C" {

FMD_API fmd_status fmd_verlet_scratch_bytes(int32_t natoms, float rc_skin, float box_L, size_t* bytes) {
  return guarded([&] {
    if (!bytes || natoms <= 0) throw Error(FMD_ERR_ARG, "bad argument");
    const VerletGeom g = verlet_geom(box_L, rc_skin);
    *bytes = verlet_carve(nullptr, natoms, g.ncell).total;
  });
}

}  // extern "C"

namespace {
void verlet_build_into(const void* pos, int32_t natoms, float box_L, const int32_t* excl_off, const int32_t* excl_list,
                       float rc_skin, int32_t max_neighbors, int32_t* neighbors, int32_t* num_neighbors,
                       const VerletScratch& s, const VerletGeom& g, int32_t* overflow_flag, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const int gr = div_up(natoms, kBlock);
    k_assign<<<gr, kBlock, 0, st>>>((const float4*)pos, s.cid, s.aid, natoms, g.inv_cell, g.nx);
    FMD_CUDA_LAUNCH();
    size_t cb = s.cub_bytes;
    FMD_CUDA(cub::DeviceRadixSort::SortPairs(s.cub, cb, s.cid, s.cid_sorted, s.aid, s.sorted, natoms, 0, 32, st));
    FMD_CUDA(cudaMemsetAsync(s.start, 0, sizeof(int) * g.ncell, st));
    FMD_CUDA(cudaMemsetAsync(s.end, 0, sizeof(int) * g.ncell, st));
    k_ranges<<<gr, kBlock, 0, st>>>(s.cid_sorted, s.start, s.end, natoms);
    FMD_CUDA_LAUNCH();
    const float rcs2 = rc_skin * rc_skin;
    k_build<<<gr, kBlock, 0, st>>>((const float4*)pos, s.sorted, s.cid_sorted, s.start, s.end, excl_off, excl_list,
                                   neighbors, num_neighbors, natoms, g.nx, rcs2, box_L, 1.0f / box_L, max_neighbors,
                                   overflow_flag);
    FMD_CUDA_LAUNCH();
}
}  // namespace

extern "C" {

FMD_API fmd_status fmd_launch_verlet_build(const void* pos, int32_t natoms, float box_L, const int32_t* excl_off,
                                           const int32_t* excl_list, float rc_skin, int32_t max_neighbors,
                                           int32_t* neighbors, int32_t* num_neighbors, void* scratch,
                                           size_t scratch_bytes, int32_t* overflow_flag, void* stream) {
  return guarded([&] {
    if (!pos || natoms <= 0 || !neighbors || !num_neighbors || !scratch || max_neighbors <= 0)
      throw Error(FMD_ERR_ARG, "bad argument");
    const VerletGeom g = verlet_geom(box_L, rc_skin);
    const VerletScratch s = verlet_carve(scratch, natoms, g.ncell);
    if (s.total > scratch_bytes) throw Error(FMD_ERR_ARG, "scratch buffer too small");
    verlet_build_into(pos, natoms, box_L, excl_off, excl_list, rc_skin, max_neighbors, neighbors, num_neighbors, s, g,
                      overflow_flag, stream);
  });
}

// Same result as fmd_launch_verlet_build, with the scratch in the library's
// static device array instead of caller memory; allocates nothing.
FMD_API fmd_status fmd_launch_verlet_build_static(const void* pos, int32_t natoms, float box_L,
                                                  const int32_t* excl_off, const int32_t* excl_list, float rc_skin,
                                                  int32_t max_neighbors, int32_t* neighbors, int32_t* num_neighbors,
                                                  int32_t* overflow_flag, void* stream) {
  return guarded([&] {
    if (!pos || natoms <= 0 || !neighbors || !num_neighbors || max_neighbors <= 0)
      throw Error(FMD_ERR_ARG, "bad argument");
    if (natoms > kStaticMaxAtoms)
      throw Error(FMD_ERR_CAPACITY, "natoms exceeds the static-scratch limit of " + std::to_string(kStaticMaxAtoms));
    if (!(std::isfinite(box_L) && std::isfinite(rc_skin) && box_L > 0.0f && rc_skin > 0.0f))
      throw Error(FMD_ERR_ARG, "box_L and rc_skin must be finite and positive");
    // at most 40 cells per axis (40^3 = 64000 <= kStaticMaxCells), checked
    // before the cell count is formed
    if (box_L / rc_skin >= (float)(kStaticMaxCellsPerAxis + 1))
      throw Error(FMD_ERR_CAPACITY, "cell grid exceeds the static-scratch limit of " +
                                        std::to_string(kStaticMaxCellsPerAxis) + " cells per axis");
    const VerletGeom g = verlet_geom(box_L, rc_skin);
    if (g.ncell > kStaticMaxCells)
      throw Error(FMD_ERR_CAPACITY, "cell grid exceeds the static-scratch limit of " + std::to_string(kStaticMaxCells) +
                                        " cells");
    void* base = static_scratch_for_current_device();
    const VerletScratch s = verlet_carve(base, natoms, g.ncell);
    if (s.total > kStaticScratchBytes) throw Error(FMD_ERR_CAPACITY, "problem too large for the static scratch");
    verlet_build_into(pos, natoms, box_L, excl_off, excl_list, rc_skin, max_neighbors, neighbors, num_neighbors, s, g,
                      overflow_flag, stream);
  });
}

FMD_API fmd_status fmd_launch_lj(const void* pos, void* force, float* virial, const void* lj_params,
                                 const int32_t* neighbors, const int32_t* num_neighbors, int32_t natoms, int32_t ntypes,
                                 float rc2, float box_L, float inv_L, void* stream) {
  return guarded([&] {
    if (!pos || !force || !virial || !lj_params || !neighbors || !num_neighbors || natoms <= 0 || ntypes <= 0)
      throw Error(FMD_ERR_ARG, "bad argument");
    k_lj<<<div_up(natoms, kBlock), kBlock, 0, (cudaStream_t)stream>>>(
        (const float4*)pos, (float4*)force, virial, (const float2*)lj_params, neighbors, num_neighbors, natoms,
        ntypes, rc2, box_L, inv_L);
    FMD_CUDA_LAUNCH();
  });
}

FMD_API fmd_status fmd_tile_list_scratch_bytes(int32_t natoms, size_t* bytes) {
  return guarded([&] {
    if (!bytes || natoms <= 0) throw Error(FMD_ERR_ARG, "bad argument");
    *bytes = tile_carve(nullptr, (natoms + 31) / 32).total;
  });
}

FMD_API fmd_status fmd_launch_tile_list(const void* pos, int32_t natoms, float box_L, float rc_skin, int32_t* offsets,
                                        int32_t* neighbors, int32_t capacity, int32_t* npairs, void* scratch,
                                        size_t scratch_bytes, void* stream) {
  return guarded([&] {
    if (!pos || natoms <= 0 || !offsets || capacity < 0 || (capacity > 0 && !neighbors) || !scratch)
      throw Error(FMD_ERR_ARG, "bad argument");
    if (!(std::isfinite(box_L) && std::isfinite(rc_skin) && box_L > 0.0f && rc_skin > 0.0f))
      throw Error(FMD_ERR_ARG, "box_L and rc_skin must be finite and positive");
    const int T = (natoms + 31) / 32;
    const TileScratch s = tile_carve(scratch, T);
    if (s.total > scratch_bytes) throw Error(FMD_ERR_ARG, "scratch buffer too small");
    cudaStream_t st = (cudaStream_t)stream;
    const float inv_L = 1.0f / box_L, rc2 = rc_skin * rc_skin;
    k_tile_bbox<<<T, 32, 0, st>>>((const float4*)pos, s.tmin, s.tmax, natoms);
    FMD_CUDA_LAUNCH();
    const int wpb = 4, gr = div_up(T, wpb);
    k_tile_pairs<false><<<gr, 32 * wpb, 0, st>>>(s.tmin, s.tmax, T, box_L, inv_L, rc2, s.cnt, nullptr, nullptr, 0);
    FMD_CUDA_LAUNCH();
    size_t cb = s.cub_bytes;
    FMD_CUDA(cub::DeviceScan::ExclusiveSum(s.cub, cb, s.cnt, offsets, T + 1, st));
    k_tile_pairs<true><<<gr, 32 * wpb, 0, st>>>(s.tmin, s.tmax, T, box_L, inv_L, rc2, nullptr, offsets, neighbors,
                                                capacity);
    FMD_CUDA_LAUNCH();
    if (npairs) {
      FMD_CUDA(cudaMemcpyAsync(npairs, offsets + T, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      FMD_CUDA(cudaStreamSynchronize(st));
      if (*npairs > capacity) throw Error(FMD_ERR_OVERFLOW, "tile pairs exceed the capacity");
    }
  });
}

FMD_API fmd_status fmd_launch_lj_tiles(const void* pos, void* force, float* virial, const void* lj_params,
                                       const int32_t* tile_offsets, const int32_t* tile_neighbors,
                                       const int32_t* exclusion_offsets, const int32_t* exclusion_list,
                                       int32_t natoms, int32_t ntypes, float rc2, float box_L, float inv_L,
                                       void* stream) {
  return guarded([&] {
    if (!pos || !force || !virial || !lj_params || !tile_offsets || !tile_neighbors || natoms <= 0 || ntypes <= 0)
      throw Error(FMD_ERR_ARG, "bad argument");
    if (!exclusion_offsets != !exclusion_list) throw Error(FMD_ERR_ARG, "exclusion offsets and list go together");
    const int T = (natoms + 31) / 32;
    k_lj_tiles<<<div_up(T, kTileWarps), 32 * kTileWarps, 0, (cudaStream_t)stream>>>(
        (const float4*)pos, (float4*)force, virial, (const float2*)lj_params, tile_offsets, tile_neighbors,
        exclusion_offsets, exclusion_list, natoms, T, ntypes, rc2, box_L, inv_L);
    FMD_CUDA_LAUNCH();
  });
}

FMD_API fmd_status fmd_morton_scratch_bytes(int32_t natoms, size_t* bytes) {
  return guarded([&] {
    if (!bytes || natoms <= 0) throw Error(FMD_ERR_ARG, "bad argument");
    *bytes = morton_carve(nullptr, natoms).total;
  });
}

FMD_API fmd_status fmd_launch_morton_sort(void* pos, void* vel, int32_t natoms, float inv_L, int32_t* perm,
                                          void* scratch, size_t scratch_bytes, void* stream) {
  return guarded([&] {
    if (!pos || natoms <= 0 || !perm || !scratch) throw Error(FMD_ERR_ARG, "bad argument");
    MortonScratch s = morton_carve(scratch, natoms);
    if (s.total > scratch_bytes) throw Error(FMD_ERR_ARG, "scratch buffer too small");
    cudaStream_t st = (cudaStream_t)stream;
    const int gr = div_up(natoms, kBlock);
    k_morton_keys<<<gr, kBlock, 0, st>>>((const float4*)pos, s.keys, s.idx, natoms, inv_L);
    FMD_CUDA_LAUNCH();
    size_t cb = s.cub_bytes;
    FMD_CUDA(cub::DeviceRadixSort::SortPairs(s.cub, cb, s.keys, s.keys_sorted, s.idx, perm, natoms, 0, 30, st));
    k_gather4<<<gr, kBlock, 0, st>>>(s.tmp, (const float4*)pos, perm, natoms);
    FMD_CUDA_LAUNCH();
    FMD_CUDA(cudaMemcpyAsync(pos, s.tmp, sizeof(float4) * natoms, cudaMemcpyDeviceToDevice, st));
    if (vel) {
      k_gather4<<<gr, kBlock, 0, st>>>(s.tmp, (const float4*)vel, perm, natoms);
      FMD_CUDA_LAUNCH();
      FMD_CUDA(cudaMemcpyAsync(vel, s.tmp, sizeof(float4) * natoms, cudaMemcpyDeviceToDevice, st));
    }
  });
}

}  // extern "C"
