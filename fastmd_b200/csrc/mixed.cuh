// Mixed-precision batched engine: device data layout shared by the kernels
// (mixed_kernels.cu) and the host batch manager (batch.cpp).
//
// Layout in HBM.  Replicas occupy disjoint slot segments of the batch arrays;
// a replica's segment is padded to a multiple of kChunk slots so that no block
// (one chunk) straddles two replicas, which makes every per-replica reduction
// independent of what else is in the batch.
//
//   pos[s]   float4 {ox, oy, oz, packed}   offset from the atom's cell corner
//                                          (absolute units) + cell (9 bits per
//                                          axis) and type (5 bits) in .w
//   vel[s]   float4 {vx, vy, vz, 1/m}
//   force[s] float4 {fx, fy, fz, pe_i}
//   ref[s]   float4 offsets at the last rebuild (displacement test); .w = atom id
//   img[s]   int4   {ix, iy, iz, atom id}  image flags + replica-local atom id
//   nbr      uint32 per (tile, k, lane): replica-local slot of j (22 bits) and
//            the periodic shift of j relative to i as three 3-bit axis codes
//            above it (see entry_code below)
//
// A position is r = (c + 0) * h + o with h = L / G the cell edge; pair
// displacements are formed as (o_i - o_j) - e * h, so their precision is set by
// the cell edge, not by the box size.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "nhc.h"

namespace fmd {
namespace mixed {

constexpr int kChunk = 128;       // slots per block / per reduction partial
constexpr int kTile = 32;         // slots per warp tile
constexpr int kMaxTypes = 16;
constexpr int kMaxTables = 8;  // distinct pair tables per replica
constexpr int kGhostType = 31;
constexpr int kMaxG = 512;        // cells per axis (9 bits)
// Neighbor-list entry: slot (22 bits) | ax << 22 | ay << 25 | az << 28.  The
// three axis codes name one of 125 periodic shift vectors: per axis a in 0..4
// for e*h + k*dL with (e, k) = (-1,-1), (-1,0), (0,0), (1,0), (1,1).  The
// vector is the same for every atom of a replica.  Each code sits in a field
// of its own, so a force loop reads it with one bit-field extract.
constexpr int kSlotBits = 22;
constexpr uint32_t kIdxMask = (1u << kSlotBits) - 1;
constexpr int kShiftCodes = 125;  // 25 ax + 5 ay + az: the index into a table of all 125 vectors
__host__ __device__ inline uint32_t entry_code(int ax, int ay, int az) {
  return ((uint32_t)ax << kSlotBits) | ((uint32_t)ay << (kSlotBits + 3)) | ((uint32_t)az << (kSlotBits + 6));
}
__host__ __device__ inline int entry_ax(uint32_t w) { return (int)((w >> kSlotBits) & 7u); }
__host__ __device__ inline int entry_ay(uint32_t w) { return (int)((w >> (kSlotBits + 3)) & 7u); }
__host__ __device__ inline int entry_az(uint32_t w) { return (int)(w >> (kSlotBits + 6)); }
// Lists are padded to a multiple of kListPad entries with the atom's own
// slot and the shift (h + dL) on every axis (codes 4, 4, 4: (e, k) = (1, 1)), so
// the force loop runs whole batches and a padding entry lies sqrt(3) (h + dL)
// > rc away: the cutoff test alone gives it an exact zero.  (The cell edge h
// is at least rc + skin at a rebuild; an NPT contraction shrinks it by at
// most rc / (rc + skin) before the rebuild trigger fires, so h >= rc.)
constexpr uint32_t kPadBits = (4u << kSlotBits) | (4u << (kSlotBits + 3)) | (4u << (kSlotBits + 6));
constexpr int kListPad = 8;
constexpr int kPrunePad = 4;  // the pruned list: padded to whole force batches only
constexpr double kPruneDelta = 0.12;  // pruned-list margin beyond rc (sigma)
constexpr int32_t kNoForcedRebuild = 1 << 30;  // rebuild cadence: skin trigger only
constexpr uint32_t kSlotMask26 = (1u << 26) - 1;  // bonded-table slot field
constexpr int kNumPartials = 14;  // pe, vir[6], ke[6], sum m v^2
constexpr int kMaxBondsPerAtom = 4;   // per-slot bonded tables rebuilt with the list
constexpr int kMaxAnglesPerAtom = 8;

enum Mode : int32_t { kModeRun = 0, kModePushoff = 1 };

// Per-kernel launch counters (executed launches, graph conditionals included).
enum KernelKind : int {
  kKPre = 0, kKBin, kKScan, kKScatter, kKCellsort, kKPermute, kKTopo, kKNeighbors, kKForce, kKForceEv, kKPost,
  kKPlan, kKCommit, kKTable, kKernelKinds
};

// Per-replica record (device).  Static fields are set at admission; dynamic
// ones are updated by the kernels.
// Per-step scalars of a replica's pre-force update: thermostat / barostat
// factors for the step about to be taken.  Computed once per replica (by the
// last block of the previous post-force) and read by every block.
struct StepScalars {
  int adv;
  int64_t step;  // step being taken (1-based)
  float hdt, dt;
  float c1;      // Langevin velocity decay
  float c2kT;    // c2 * sqrt(kT) (per-type mass applied per atom)
  float vscale;  // velocity scale applied before the kick (pending post * pre)
  float ev, fpos;       // NPT: position scale and drift factor
  float dh;             // NPT: c * dh term (h_old * ev - h_new)
  float h_new;          // NPT: new cell edge
  float h_old, inv_Lold;  // NPT: frame of the stored positions
  float dW;             // NPT: L_new - L_old * ev, applied per wrapped period
  uint32_t stream;
  int ens;
  NHScalars nh;         // updated chain / barostat state (committed by the last block)
  double L_new;
};

struct Rep {
  // --- static
  int32_t active;
  int32_t slot_base, slot_cap, natoms;
  int32_t chunk_base, nchunks;
  int32_t cell_base, P;          // Morton-keyed cell arrays: P^3 entries (P = pow2 >= G_alloc)
  int32_t G_alloc;
  int64_t nbr_base;              // first list entry of the replica's first tile
  int32_t M;                     // list capacity per atom
  int32_t bond_base, angle_base; // CSR entry bases
  int32_t ntypes;
  int32_t ensemble;
  int32_t chain_M;
  int32_t chain_carry;           // run.conf nh_chain_carry: chain accelerations kept between half steps
  int32_t max_between;           // forced rebuild cadence (steps; kNoForcedRebuild: skin trigger only)
  int64_t nsteps;                // run.conf nsteps (ramp denominator)
  uint64_t seed;
  double dt, rc, skin;
  double T0, T1, Tdamp, P0, P1, Pdamp;
  double c1;                     // exp(-dt / Tdamp)
  double Q1, Qr, W, V0;
  float invm[kMaxTypes];
  float lj_eps24[kMaxTypes * kMaxTypes];  // 24 eps
  float lj_sig2[kMaxTypes * kMaxTypes];   // sig^2
  float fene[4 * 4];             // up to 4 bond types: k, R0^2, eps, sig^2
  float angp[2 * 4];             // up to 4 angle types: k, theta0
  // tabulated pair potentials (force/table.cu): table per type pair (-1:
  // none), grid of each table, its points at Dev::tab + tab_off (force, energy)
  int32_t ntables;
  int8_t table_of[kMaxTypes * kMaxTypes];
  float tab_rmin[kMaxTables], tab_rmax[kMaxTables], tab_dr[kMaxTables], tab_inv_dr[kMaxTables];
  int32_t tab_n[kMaxTables], tab_off[kMaxTables];
  // --- dynamic
  int32_t mode;
  double fcap;                   // force cap (push-off)
  double push_dt;
  int64_t step, stop_step;
  int32_t since, rebuild_now, adv;
  int32_t G;
  double L;      // box edge (barostat value)
  double Lpos;   // box the stored positions are wrapped in (last pre-force)
  double L_list; // box the neighbor list was built in (box-shrink term of the rebuild trigger)
  double list_scale;  // product of the NPT position scale factors since the list was built
  double L_filter;    // box, and product of the position scale factors, since the pruned
  double filter_scale;  // list was last filtered (its own box-shrink term)
  float h;
  uint32_t maxdisp_bits;
  // Pruned list: the pairs of the rc + skin list within rc + prune_delta,
  // walked by the force kernels instead of the full list.  It is re-filtered
  // when a displacement since the last filter exceeds prune_delta / 2; ref
  // then holds the positions of the last filter (or rebuild), and disp_acc
  // the sum of the largest displacements of the filters since the rebuild,
  // so that largest displacement since the last filter + disp_acc bounds
  // every displacement since the rebuild (the full list's trigger).  Under
  // NPT the filter's trigger takes the contraction since the filter into
  // account as the rebuild's does (L_filter, filter_scale).
  // prune_delta = 0: no pruned list.
  float prune_delta;
  float disp_acc;
  int32_t status;
  int64_t rebuilds;
  NHScalars nh;
  double pending_scale;          // NH post-force velocity scale applied at the next pre-force
  // reductions of the last completed step
  double pe, vir[6], ke[6];
  int64_t thermo_step;
  int32_t thermo_freq;           // run.conf thermo cadence (0: off); energies/virial computed on those steps
  int32_t stress_freq;           // run.conf stress cadence (0: off); a pressure-tensor sample feeds the correlator
  int32_t force_ev;              // host request: compute energies/virial at the next force evaluation
  int64_t ev_step;               // step whose energies/virial are in pe/vir
  int32_t defer;                 // this step's post-force kick is applied by the next pre-force
  StepScalars next;              // scalars of the next pre-force (valid when next_valid)
  int32_t next_valid;            // cleared by every host upload and by each pre-force
};

// Energies and virial are needed on thermo steps, for NPT (the barostat uses
// the virial every step) and when the host asks for them.
__host__ __device__ inline bool stress_step(const Rep& R) {
  return R.mode != kModePushoff && R.stress_freq > 0 && (R.step % R.stress_freq) == 0;
}

__host__ __device__ inline bool need_ev(const Rep& R) {
  if (R.force_ev) return true;
  if (R.mode != kModePushoff && R.ensemble == FMD_NPT_NH) return true;
  if (stress_step(R)) return true;
  return R.thermo_freq > 0 && (R.step % R.thermo_freq) == 0;
}

// Multiple-tau stress autocorrelator per replica (analysis/correlator.cu
// semantics: kAcfLevels levels of kAcfPoints samples of the 6 pressure
// components, each level fed with block averages of kAcfPoints samples of
// the level below).  FP64 state, kAcfWords doubles per replica:
constexpr int kAcfLevels = 16, kAcfPoints = 16, kAcfComps = 6;
constexpr int kAcfBuf = 0;                                              // [level][point][comp] samples
constexpr int kAcfCorr = kAcfBuf + kAcfLevels * kAcfPoints * kAcfComps;  // [level][lag][comp] sums of products
constexpr int kAcfCnt = kAcfCorr + kAcfLevels * kAcfPoints * kAcfComps;  // [level][lag] products summed
constexpr int kAcfIdx = kAcfCnt + kAcfLevels * kAcfPoints;               // [level] insert position
constexpr int kAcfAcc = kAcfIdx + kAcfLevels;                            // [level][comp] block accumulator
constexpr int kAcfAccN = kAcfAcc + kAcfLevels * kAcfComps;               // [level] samples in the block
constexpr int kAcfWords = kAcfAccN + kAcfLevels;

// Device pointers of the batch arrays.
struct Dev {
  Rep* reps;
  const int4* chunk_rep;         // per chunk: replica (-1 free), first slot, atoms in it, index in the replica
  float4* pos;
  float4* vel;
  float4* force;
  float4* ref;
  int4* img;
  // rebuild scratch
  float4* tpos;
  int4* timg;
  float4* tvel;
  uint32_t* key;                 // cell key per slot during a rebuild
  int32_t* perm;                 // new local slot -> old local slot
  int32_t* bucket;               // cell bucket (old local slots)
  int32_t* cell_cnt;             // per cell key
  int32_t* cell_start;
  int32_t* cell_fill;
  // id-indexed (slot_base + atom id)
  int32_t* slot_of;
  int32_t* boff;                 // bond CSR offsets (natoms + 1 per replica, relative to bond_base)
  int32_t* aoff;                 // angle CSR offsets
  // topology entries
  int2* bent;                    // {partner id, type | first << 8}
  int4* aent;                    // {i id, j id, k id, type | role << 8}
  // per-slot bonded tables (rebuilt with the list): partner slots and roles
  int32_t* tcnt;                 // bonds | angles << 8
  uint32_t* bnd;                 // [slot * kMaxBondsPerAtom]: partner slot | type << 26 | first << 30
  uint2* ang;                    // [slot * kMaxAnglesPerAtom]: {other1 | role << 26, other2 | type << 26}
  // neighbor list
  uint32_t* nbr;
  int32_t* ncnt;
  uint32_t* pnbr;                // pruned list (same layout and bases as nbr)
  int32_t* pcnt;
  double* part;                  // [kNumPartials][part_stride]: value q of chunk c at q * part_stride + c
  int64_t part_stride;           // chunks allocated
  double* acf;                   // [replica][kAcfWords] stress autocorrelator state
  const float2* tab;             // pair-table points (force, energy) of every replica's tables
  unsigned long long* kcount;    // [kKernelKinds] launches executed (block 0 of each launch counts)
  // rebuild work list: header (RbHeader), rb_cap replicas, then three
  // offset arrays of rb_cap + 1 (chunk items, cell-group items, home-cell
  // items)
  int* rb;
  int rb_cap;
};

// Axis part of the shift code for cell shift e and wrap count k; -1 when
// (e, k) is not one of the five representable cases.
__host__ __device__ inline int axis_shift_code(int e, int k) {
  if (e == 0) return k == 0 ? 2 : -1;
  if (e == -1) return k == -1 ? 0 : (k == 0 ? 1 : -1);
  if (e == 1) return k == 1 ? 4 : (k == 0 ? 3 : -1);
  return -1;
}
__host__ __device__ inline int axis_code_e(int a) { return a < 2 ? -1 : (a == 2 ? 0 : 1); }
__host__ __device__ inline int axis_code_k(int a) { return a == 0 ? -1 : (a == 4 ? 1 : 0); }

__host__ __device__ inline uint32_t spread3(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ inline uint32_t cell_key(int x, int y, int z) {
  return spread3((uint32_t)x) | (spread3((uint32_t)y) << 1) | (spread3((uint32_t)z) << 2);
}
__host__ __device__ inline float pack_w(int cx, int cy, int cz, int type) {
  uint32_t u = (uint32_t)cx | ((uint32_t)cy << 9) | ((uint32_t)cz << 18) | ((uint32_t)type << 27);
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ inline uint32_t w_bits(float w) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(w);
#else
  uint32_t u;
  __builtin_memcpy(&u, &w, 4);
  return u;
#endif
}
__host__ __device__ inline int w_cx(uint32_t u) { return (int)(u & 511u); }
__host__ __device__ inline int w_cy(uint32_t u) { return (int)((u >> 9) & 511u); }
__host__ __device__ inline int w_cz(uint32_t u) { return (int)((u >> 18) & 511u); }
__host__ __device__ inline int w_type(uint32_t u) { return (int)(u >> 27); }

// Kernel launchers (mixed_kernels.cu).
// Conditional-node handles of one captured step (CUDA graph IF nodes around
// the rebuild and the two force-kernel variants); set from the device by the
// pre-force kernel.  use == 0 outside a graph (every kernel launched, blocks
// of replicas that need no work return at once).
struct StepConds {
  int use;
  cudaGraphConditionalHandle rebuild, rebuild_full, force_plain, force_ev, post, prune;  // force_plain: unused (plain node)
};

// Rebuild work list header (ints at the front of Dev::rb).
// The work list holds the replicas that rebuild this step (rebuild_now = 1)
// and those that only re-filter their pruned list (rebuild_now = 2);
// kRbRebuilds counts the former.
enum RbHeader : int { kRbCount = 0, kRbCommits = 1, kRbMode = 2, kRbRebuilds = 3, kRbHead = 4 };
constexpr int kRbOffArrays = 4;  // chunk items (rebuilding), cell groups, home cells, chunk items (all listed)
enum RbMode : int { kRbNone = 0, kRbList = 1, kRbFull = 2, kRbPrune = 3 };  // kRbPrune: list filters only
constexpr int kRbFullMin = 8;  // replicas rebuilding in one step before full grids pay

// Launch geometry of a step for the current batch layout.
struct StepShape {
  int nchunks, nreps;   // chunk blocks, replica-indexed blocks
  int max_cells;        // largest P^3 (Morton cells) over replicas
  int max_home;         // largest G_alloc^3 (home cells) over replicas
  int force_variant, nbr_variant;
  int has_table;        // some replica has tabulated pairs: the table pass follows the forces
};
using RebuildShape = StepShape;
constexpr int kForceVariants = 15;
constexpr int kNbrVariants = 3;
// One step with direct launches.  The rebuild form is read back from the
// device after the per-replica commits (one small host read per step).
void launch_step(const Dev& d, const StepShape& g, int* host_mode, cudaStream_t st);
// The same step recorded into the graph being captured on st, with the
// conditional nodes; side is a second stream used to capture their bodies.
// st2: a second capture stream for the parallel branches of a step.
// Records one step into the graph being captured on st.  side / side_hi
// record conditional-node bodies (side_hi: high priority, for the rebuild
// branches); br: four further streams for the parallel branches.
void capture_step(const Dev& d, const StepShape& g, cudaStream_t st, cudaStream_t side, cudaStream_t side_hi,
                  const cudaStream_t* br);
// filter: also filter the rebuilt replicas' pruned lists (k_prune); the step
// leaves that to the work-list force launch that follows.
void launch_rebuild_full(const Dev& d, const RebuildShape& g, cudaStream_t st, bool filter = true);
void launch_force(const Dev& d, int nchunks, bool ev, int variant, cudaStream_t st, bool skip_rebuilt);
// Positions (3 floats per atom, id order) of replica r, wrapped in its
// last pre-force box, into out.
void launch_pack_frame(const Dev& d, int r, int natoms, float* out, cudaStream_t st);
// Work-list offsets of the listed replicas (a step where none rebuilds).
void launch_rb_plan(const Dev& d, cudaStream_t st);
// Filters of the listed replicas' pruned lists after their plan, without a
// force evaluation (host calls).
void launch_prune_only(const Dev& d, cudaStream_t st);
// Forces of the replicas on the rebuild work list (after their rebuild),
// with the filter of their pruned lists.
void launch_force_rebuilt(const Dev& d, bool ev, int variant, cudaStream_t st);
// Rebuild of the replicas on the work list (rb): bin, scan, scatter, cell sort,
// permute, bonded tables, neighbor lists (and, filter, their pruned lists).
void launch_rebuild(const Dev& d, int nreps, int nbr_variant, cudaStream_t st, bool filter = true);
void launch_forces_only(const Dev& d, int nchunks, int variant, bool has_table, cudaStream_t st);
// Tabulated pairs of the replicas that have them, added to the forces (and,
// ev, to the energies and virial partials) the force kernel wrote.  sel: 0
// every replica, 1 replicas not rebuilding this step, 2 rebuilding ones.
void launch_table(const Dev& d, int nchunks, bool ev, int sel, cudaStream_t st);
void launch_reduce_only(const Dev& d, int nchunks, int nreps, cudaStream_t st, int mode);
// Scalars of the next pre-force for replicas whose copy a host upload made stale.
void launch_prepare(const Dev& d, int nreps, cudaStream_t st);  // 0 setup, 2 re-evaluation

}  // namespace mixed
}  // namespace fmd
