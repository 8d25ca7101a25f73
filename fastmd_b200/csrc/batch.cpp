// Host side of the mixed-precision batched engine: admission of replicas into
// the segmented batch arrays, the CUDA-graph step loop, readout, and the C ABI
// for batches.  The single-system mixed form (fmd_sim with FMD_FORM_MIXED) is a
// batch holding one replica.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <vector>

#include "batch.h"
#include "dev_common.cuh"
#include "engine.h"
#include "mixed.cuh"

namespace fmd {
namespace mixed {

// ------------------------------------------------------------- allocator
int64_t SegAlloc::alloc(int64_t n) {
  if (n <= 0) n = 1;
  for (auto it = free_.begin(); it != free_.end(); ++it) {
    if (it->second >= n) {
      const int64_t at = it->first;
      const int64_t rest = it->second - n;
      free_.erase(it);
      if (rest > 0) free_[at + n] = rest;
      used_[at] = n;
      hwm_ = std::max(hwm_, at + n);
      return at;
    }
  }
  return -1;
}

void SegAlloc::release(int64_t at) {
  auto u = used_.find(at);
  if (u == used_.end()) return;
  int64_t start = at, len = u->second;
  used_.erase(u);
  auto nx = free_.lower_bound(start);
  if (nx != free_.end() && nx->first == start + len) {
    len += nx->second;
    nx = free_.erase(nx);
  }
  if (nx != free_.begin()) {
    auto pv = std::prev(nx);
    if (pv->first + pv->second == start) {
      start = pv->first;
      len += pv->second;
      free_.erase(pv);
    }
  }
  free_[start] = len;
  hwm_ = 0;
  for (auto& kv : used_) hwm_ = std::max(hwm_, kv.first + kv.second);
}

static float uint_as_float_host(uint32_t u) {
  float f;
  std::memcpy(&f, &u, sizeof f);
  return f;
}

// ------------------------------------------------------------- sizing
static int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

ReplicaPlan plan_replica(const RunConfig& cfg, int32_t natoms, double L) {
  ReplicaPlan p;
  const double rcs = cfg.rc + cfg.skin;
  const double grow = (cfg.ensemble == FMD_NPT_NH) ? 1.3 : 1.0;
  int G = (int)std::floor(grow * L / (rcs * 1.0001));
  if (G < 1) G = 1;
  if (G > kMaxG) throw Error(FMD_ERR_CONFIG, "box too large for the cell grid (more than 512 cells per axis)");
  p.G_alloc = G;
  p.P = next_pow2(G);
  p.ncell = (int64_t)p.P * p.P * p.P;
  p.slot_cap = ((natoms + 1 + kChunk - 1) / kChunk) * kChunk;
  p.nchunks = p.slot_cap / kChunk;
  const double rho = natoms / (L * L * L);
  const double expect = rho * (4.0 / 3.0) * 3.14159265358979323846 * rcs * rcs * rcs;
  int M = (int)std::ceil(1.5 * expect + 32.0);
  M = ((M + 31) / 32) * 32;
  p.M = std::max(64, M);
  p.nbr_entries = (int64_t)(p.slot_cap / kTile) * p.M * kTile;
  return p;
}

int64_t bytes_per_slot() {
  return 6 * 16 + 2 * 16 + 9 * 4 + kMaxBondsPerAtom * 4 + kMaxAnglesPerAtom * 8 +
         (int64_t)(kNumPartials * 8) / kChunk + 1;
}

int64_t estimate_bytes(const ReplicaPlan& p, int32_t nbonds, int32_t nangles) {
  return p.slot_cap * bytes_per_slot() + p.nbr_entries * 8 + p.ncell * 12 + (int64_t)2 * nbonds * 8 +
         (int64_t)3 * nangles * 16 + (int64_t)sizeof(Rep);
}

// ------------------------------------------------------------- batch
Batch::Batch(const fmd_batch_opts& o, const BatchCaps* exact) {
  device_ = o.device;
  FMD_CUDA(cudaSetDevice(device_));
  FMD_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  FMD_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  for (auto& b : branch_) FMD_CUDA(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
  {
    int least = 0, greatest = 0;
    FMD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    FMD_CUDA(cudaStreamCreateWithPriority(&side_hi_, cudaStreamNonBlocking, greatest));
  }
  // graph_steps < 0: no graph (every step launched directly; for profilers
  // that cannot see into graphs with conditional nodes)
  graph_steps_ = o.graph_steps > 0 ? o.graph_steps : (o.graph_steps < 0 ? 0 : 50);
  max_reps_ = o.max_replicas > 0 ? o.max_replicas : 256;
  BatchCaps c;
  if (exact) {
    c = *exact;
  } else {
    const double budget = (o.hbm_budget_gb > 0 ? o.hbm_budget_gb : 150.0) * 1e9;
    int64_t slots = o.max_atoms > 0 ? o.max_atoms : (int64_t)4 << 20;
    // list entries at ~160 per atom, cells at ~4 per atom (Morton padding), topology at ~3 per atom
    int64_t per = bytes_per_slot() + 2 * 160 * 4 + 4 * 12 + 3 * 16;  // full and pruned lists
    slots = std::min<int64_t>(slots, (int64_t)(budget / per));
    slots = ((slots + kChunk - 1) / kChunk) * kChunk;
    c.slots = slots;
    c.nbr = slots * 160;
    c.cells = slots * 4 + 4096;
    c.bonds = slots * 3;
    c.angles = slots * 4;
  }
  caps_ = c;
  budget_bytes_ = (int64_t)((o.hbm_budget_gb > 0 ? o.hbm_budget_gb : 150.0) * 1e9);
  slot_alloc_.reset(c.slots / kChunk);
  cell_alloc_.reset(c.cells);
  nbr_alloc_.reset(c.nbr / 1024);  // 1024-entry units
  bond_alloc_.reset(c.bonds);
  angle_alloc_.reset(c.angles);
  const size_t S = (size_t)c.slots;
  pos_.alloc_zero(S);
  vel_.alloc_zero(S);
  force_.alloc_zero(S);
  ref_.alloc_zero(S);
  img_.alloc_zero(S);
  tpos_.alloc(S);
  timg_.alloc(S);
  tvel_.alloc(S);
  key_.alloc(S);
  perm_.alloc(S);
  bucket_.alloc(S);
  slot_of_.alloc_zero(S);
  boff_.alloc_zero(S);
  aoff_.alloc_zero(S);
  ncnt_.alloc_zero(S);
  pcnt_.alloc_zero(S);
  tcnt_.alloc_zero(S);
  bnd_.alloc(S * kMaxBondsPerAtom);
  ang_.alloc(S * kMaxAnglesPerAtom);
  part_.alloc_zero(S / kChunk * kNumPartials);
  kcount_.alloc_zero(kKernelKinds);
  acf_.alloc_zero((size_t)max_reps_ * kAcfWords);
  rb_.alloc_zero(kRbHead + (size_t)max_reps_ + kRbOffArrays * ((size_t)max_reps_ + 1));
  cell_cnt_.alloc_zero(c.cells);
  cell_start_.alloc_zero(c.cells);
  cell_fill_.alloc_zero(c.cells);
  bent_.alloc(std::max<int64_t>(1, c.bonds));
  aent_.alloc(std::max<int64_t>(1, c.angles));
  nbr_.alloc(c.nbr);
  pnbr_.alloc(c.nbr);
  reps_.alloc_zero(max_reps_);
  chunk_rep_.alloc(S / kChunk);
  slot_cap_chunks_ = (int)(S / kChunk);
  h_chunk_rep_.assign(S / kChunk, make_int4(-1, 0, 0, 0));
  FMD_CUDA(cudaMemcpy(chunk_rep_, h_chunk_rep_.data(), h_chunk_rep_.size() * sizeof(int4), cudaMemcpyHostToDevice));
  h_reps_.assign(max_reps_, Rep{});
  info_.resize(max_reps_);
  bytes_ = (int64_t)S * bytes_per_slot() + c.nbr * 4 + c.cells * 12 + c.bonds * 8 + c.angles * 16;
}

Batch::~Batch() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  if (st_) cudaStreamDestroy(st_);
  if (side_) cudaStreamDestroy(side_);
  for (auto& b : branch_)
    if (b) cudaStreamDestroy(b);
  if (side_hi_) cudaStreamDestroy(side_hi_);
}

Dev Batch::dev() const {
  Dev d;
  d.reps = reps_;
  d.chunk_rep = chunk_rep_;
  d.pos = pos_;
  d.vel = vel_;
  d.force = force_;
  d.ref = ref_;
  d.img = img_;
  d.tpos = tpos_;
  d.timg = timg_;
  d.tvel = tvel_;
  d.key = key_;
  d.perm = perm_;
  d.bucket = bucket_;
  d.cell_cnt = cell_cnt_;
  d.cell_start = cell_start_;
  d.cell_fill = cell_fill_;
  d.slot_of = slot_of_;
  d.boff = boff_;
  d.aoff = aoff_;
  d.bent = bent_;
  d.aent = aent_;
  d.nbr = nbr_;
  d.ncnt = ncnt_;
  d.pnbr = pnbr_;
  d.pcnt = pcnt_;
  d.tcnt = tcnt_;
  d.bnd = bnd_;
  d.ang = ang_;
  d.part = part_;
  d.part_stride = caps_.slots / kChunk;
  d.kcount = kcount_;
  d.acf = acf_;
  d.tab = tab_.p;
  d.rb = rb_;
  d.rb_cap = max_reps_;
  return d;
}

void Batch::download_reps() {
  FMD_CUDA(cudaMemcpyAsync(h_reps_.data(), reps_, sizeof(Rep) * max_reps_, cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
}

void Batch::upload_reps() {
  // a host change may touch any input of the precomputed step scalars:
  // recompute them once per replica on the device
  for (int r = 0; r < max_reps_; ++r) h_reps_[r].next_valid = 0;
  FMD_CUDA(cudaMemcpyAsync(reps_, h_reps_.data(), sizeof(Rep) * max_reps_, cudaMemcpyHostToDevice, st_));
  launch_prepare(dev(), nreps_launch(), st_);
  FMD_CUDA_LAUNCH();
}

int Batch::nchunks_launch() const { return (int)std::max<int64_t>(1, slot_alloc_.hwm()); }
// Launch geometry: high-water marks of the layout (they only grow, so
// admitting and retiring replicas in a steady mix keeps the captured graph).
// The marks are rounded up (chunks to a multiple of 1024, replicas of 32,
// cell counts to a power of two) so that a growing mix re-captures rarely;
// blocks past the live layout return at once.
static int round_up(int x, int q) { return (x + q - 1) / q * q; }
static int pow2_at_least(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

StepShape Batch::shape() const {
  StepShape g{};
  g.nchunks = std::min(round_up(nchunks_launch(), 1024), std::max(1, slot_cap_chunks_));
  g.nreps = std::min(round_up(std::max(nreps_launch(), hw_nreps_), 32), max_reps_);
  g.max_cells = pow2_at_least(std::max(1, hw_cells_));
  g.max_home = pow2_at_least(std::max(1, hw_home_));
  g.force_variant = force_variant_;
  g.nbr_variant = nbr_variant_;
  g.has_table = 0;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && h_reps_[r].ntables > 0) g.has_table = 1;
  return g;
}
int Batch::nreps_launch() const {
  int m = 0;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used) m = r + 1;
  return std::max(1, m);
}
static void fill_static(Rep& R, const RunConfig& cfg, const Topology& t) {
  R.ntypes = cfg.ntypes;
  R.ensemble = cfg.ensemble;
  R.chain_M = cfg.chain_length;
  R.chain_carry = cfg.nh_chain_carry;
  R.max_between = 20;  // main.cu:401
  R.thermo_freq = cfg.thermo_on ? cfg.thermo_freq : 0;
  R.stress_freq = cfg.stress_on ? cfg.stress_freq : 0;
  // pruned list at rc + kPruneDelta: walked by the force kernels between
  // filters (not with a skin no wider than the margin)
  R.prune_delta = cfg.skin > kPruneDelta ? (float)kPruneDelta : 0.f;
  R.ntables = (int32_t)cfg.tables.size();
  for (int k = 0; k < kMaxTypes * kMaxTypes; ++k) R.table_of[k] = -1;
  for (size_t k = 0; k < cfg.table_of.size() && k < (size_t)(kMaxTypes * kMaxTypes); ++k)
    R.table_of[k] = (int8_t)cfg.table_of[k];
  for (int k = 0; k < R.ntables && k < kMaxTables; ++k) {
    const PairTable& tb = cfg.tables[k];
    R.tab_rmin[k] = tb.rmin;
    R.tab_rmax[k] = tb.rmax;
    R.tab_dr[k] = tb.dr;
    R.tab_inv_dr[k] = tb.inv_dr;
    R.tab_n[k] = tb.npoints;
    R.tab_off[k] = 0;  // set when the points are stored (Batch::add)
  }
  R.nsteps = cfg.nsteps;
  R.seed = cfg.seed;
  R.dt = cfg.dt;
  R.rc = cfg.rc;
  R.skin = cfg.skin;
  R.T0 = cfg.T_start;
  R.T1 = cfg.T_stop;
  R.Tdamp = cfg.Tdamp;
  R.P0 = cfg.P_start;
  R.P1 = cfg.P_stop;
  R.Pdamp = cfg.Pdamp;
  R.c1 = std::exp(-(1.0 / cfg.Tdamp) * cfg.dt);
  const double Nf = 3.0 * t.natoms, kT0 = cfg.T_start;
  R.Q1 = Nf * kT0 * cfg.Tdamp * cfg.Tdamp;
  R.Qr = kT0 * cfg.Tdamp * cfg.Tdamp;
  R.W = (Nf + 3.0) * kT0 * cfg.Pdamp * cfg.Pdamp;
  R.V0 = t.box_L * t.box_L * t.box_L;
  for (int k = 0; k < kMaxTypes; ++k) R.invm[k] = 1.0f;
  for (int k = 0; k < cfg.ntypes; ++k) R.invm[k] = (float)(1.0 / t.mass[k]);
  for (int a = 0; a < cfg.ntypes; ++a)
    for (int b = 0; b < cfg.ntypes; ++b) {
      const double eps = cfg.lj[2 * (a * cfg.ntypes + b)], sig = cfg.lj[2 * (a * cfg.ntypes + b) + 1];
      R.lj_eps24[a * cfg.ntypes + b] = (float)(24.0 * eps);
      R.lj_sig2[a * cfg.ntypes + b] = (float)(sig * sig);
    }
  if (cfg.bond.size() > 4 || cfg.angle.size() > 4)
    throw Error(FMD_ERR_CONFIG, "the mixed form supports up to 4 bond and 4 angle types");
  for (size_t k = 0; k < cfg.bond.size(); ++k) {
    R.fene[4 * k] = (float)cfg.bond[k][0];
    R.fene[4 * k + 1] = (float)(cfg.bond[k][1] * cfg.bond[k][1]);
    R.fene[4 * k + 2] = (float)cfg.bond[k][2];
    R.fene[4 * k + 3] = (float)(cfg.bond[k][3] * cfg.bond[k][3]);
  }
  for (size_t k = 0; k < cfg.angle.size(); ++k) {
    R.angp[2 * k] = (float)cfg.angle[k][0];
    R.angp[2 * k + 1] = (float)cfg.angle[k][1];
  }
}

static void init_dynamic(Rep& R, double L, int G_alloc, double rcs) {
  R.mode = kModeRun;
  R.fcap = 0;
  R.push_dt = R.dt;
  R.step = 0;
  R.stop_step = 0;
  R.since = 0;
  R.rebuild_now = 1;
  R.adv = 1;
  int G = (int)std::floor(L / (rcs * 1.0001));
  G = std::max(1, std::min(G, G_alloc));
  R.G = G;
  R.L = L;
  R.L_list = L;
  R.list_scale = 1.0;
  R.L_filter = L;
  R.filter_scale = 1.0;
  R.Lpos = L;
  R.h = (float)(L / G);
  R.maxdisp_bits = 0;
  R.disp_acc = 0.f;
  R.status = 0;
  R.rebuilds = 0;
  std::memset(&R.nh, 0, sizeof(R.nh));
  R.nh.scale = 1.0;
  R.nh.bscale = 1.0;
  R.nh.exp_vW = 1.0;
  R.nh.L = L;
  R.nh.inv_L = 1.0 / L;
  R.nh.V = L * L * L;
  R.nh.carry_dd = R.chain_carry;
  R.pending_scale = 1.0;
  R.defer = 0;
  R.force_ev = 0;
  R.ev_step = -1;
}

// Positions of atoms in data-file order into the replica's slots (slot = id);
// the first rebuild sorts them into cell order.
void Batch::upload_atoms(int r, const double* xyz, const double* vel, const int32_t* image) {
  const Rep& R = h_reps_[r];
  const ReplicaInfo& I = info_[r];
  const int n = R.natoms;
  const double L = R.L, h = R.h;
  std::vector<float4> hp(R.slot_cap), hv(R.slot_cap);
  std::vector<int4> hi(R.slot_cap);
  std::vector<int32_t> so(R.slot_cap, 0);
  for (int s = 0; s < R.slot_cap; ++s) {
    if (s < n) {
      int c[3], im[3];
      float o[3];
      for (int a = 0; a < 3; ++a) {
        double x = xyz[3 * s + a];
        const double fl = std::floor(x / L);
        x -= fl * L;
        im[a] = (image ? image[3 * s + a] : 0) + (int)fl;
        if (x >= L) {
          x -= L;
          im[a] += 1;
        }
        if (x < 0) x = 0;
        int ca = (int)std::floor(x / h);
        ca = std::max(0, std::min(ca, R.G - 1));
        c[a] = ca;
        o[a] = (float)(x - ca * h);
      }
      hp[s] = make_float4(o[0], o[1], o[2], pack_w(c[0], c[1], c[2], I.type[s]));
      hv[s] = make_float4(vel ? (float)vel[3 * s] : 0.f, vel ? (float)vel[3 * s + 1] : 0.f,
                          vel ? (float)vel[3 * s + 2] : 0.f, R.invm[I.type[s]]);
      hi[s] = make_int4(im[0], im[1], im[2], s);
      so[s] = s;
    } else {
      hp[s] = make_float4(0, 0, 0, pack_w(0, 0, 0, kGhostType));
      hv[s] = make_float4(0, 0, 0, 1.0f);
      hi[s] = make_int4(0, 0, 0, -1);
    }
  }
  const size_t b = R.slot_base;
  FMD_CUDA(cudaMemcpyAsync(pos_.p + b, hp.data(), R.slot_cap * sizeof(float4), cudaMemcpyHostToDevice, st_));
  std::vector<float4> hr(hp);
  for (int s = 0; s < R.slot_cap; ++s) {
    const int32_t id = hi[s].w;
    float idf;
    std::memcpy(&idf, &id, 4);
    hr[s].w = idf;  // the reference copy carries the atom id in .w
  }
  FMD_CUDA(cudaMemcpyAsync(ref_.p + b, hr.data(), R.slot_cap * sizeof(float4), cudaMemcpyHostToDevice, st_));
  FMD_CUDA(cudaMemcpyAsync(vel_.p + b, hv.data(), R.slot_cap * sizeof(float4), cudaMemcpyHostToDevice, st_));
  FMD_CUDA(cudaMemcpyAsync(img_.p + b, hi.data(), R.slot_cap * sizeof(int4), cudaMemcpyHostToDevice, st_));
  FMD_CUDA(cudaMemcpyAsync(slot_of_.p + b, so.data(), R.slot_cap * sizeof(int32_t), cudaMemcpyHostToDevice, st_));
  FMD_CUDA(cudaMemsetAsync(force_.p + b, 0, R.slot_cap * sizeof(float4), st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
}

int Batch::add(const RunConfig& cfg, Topology t, const fmd_melt_spec* pushoff) {
  int r = -1;
  for (int k = 0; k < max_reps_; ++k)
    if (!info_[k].used) {
      r = k;
      break;
    }
  if (r < 0) throw Error(FMD_ERR_CAPACITY, "no free replica slot");
  // neighbor-list entries address a replica's slots with 22 bits
  if ((int64_t)t.natoms + kChunk >= (int64_t)kIdxMask) throw Error(FMD_ERR_CAPACITY, "replica too large (max 4,194,000 atoms)");
  const ReplicaPlan p = plan_replica(cfg, t.natoms, t.box_L);
  const int64_t need = estimate_bytes(p, t.nbonds(), t.nangles());
  if (bytes_in_use_ + need > budget_bytes_) throw Error(FMD_ERR_CAPACITY, "device-memory budget exhausted");
  const int64_t ch = slot_alloc_.alloc(p.nchunks);
  const int64_t ce = ch >= 0 ? cell_alloc_.alloc(p.ncell) : -1;
  const int64_t nb = ce >= 0 ? nbr_alloc_.alloc((p.nbr_entries + 1023) / 1024) : -1;
  const int64_t bo = nb >= 0 ? bond_alloc_.alloc(2ll * t.nbonds()) : -1;
  const int64_t an = bo >= 0 ? angle_alloc_.alloc(3ll * t.nangles()) : -1;
  if (an < 0) {
    if (ch >= 0) slot_alloc_.release(ch);
    if (ce >= 0) cell_alloc_.release(ce);
    if (nb >= 0) nbr_alloc_.release(nb);
    if (bo >= 0) bond_alloc_.release(bo);
    throw Error(FMD_ERR_CAPACITY, "batch capacity exhausted");
  }
  ReplicaInfo& I = info_[r];
  I = ReplicaInfo{};
  I.used = true;
  I.plan = p;
  I.cfg = cfg;
  I.type = t.type;
  I.mol = t.mol;
  I.topo = t;
  I.topo.xyz.clear();
  I.topo.vel.clear();
  I.topo.image.clear();
  I.bytes = need;
  I.seg_chunk = ch;
  I.seg_cell = ce;
  I.seg_nbr = nb;
  I.seg_bond = bo;
  I.seg_angle = an;
  bytes_in_use_ += need;
  Rep& R = h_reps_[r];
  R = Rep{};
  R.active = 1;
  R.slot_base = (int32_t)(ch * kChunk);
  R.slot_cap = p.slot_cap;
  R.natoms = t.natoms;
  R.chunk_base = (int32_t)ch;
  R.nchunks = p.nchunks;
  R.cell_base = (int32_t)ce;
  R.P = p.P;
  R.G_alloc = p.G_alloc;
  R.nbr_base = nb * 1024;
  R.M = p.M;
  R.bond_base = (int32_t)bo;
  R.angle_base = (int32_t)an;
  if (cfg.tables.size() > (size_t)kMaxTables) throw Error(FMD_ERR_CONFIG, "more than 8 distinct pair tables");
  fill_static(R, cfg, t);
  init_dynamic(R, t.box_L, p.G_alloc, cfg.rc + cfg.skin);
  if (!cfg.tables.empty()) {
    // the replica's table points, appended to the batch's table array
    for (size_t k = 0; k < cfg.tables.size(); ++k) {
      R.tab_off[k] = (int32_t)tab_host_.size();
      for (int i = 0; i < cfg.tables[k].npoints; ++i)
        tab_host_.push_back(make_float2(cfg.tables[k].f[i], cfg.tables[k].e[i]));
    }
    if (tab_host_.size() > tab_.n) {
      FMD_CUDA(cudaStreamSynchronize(st_));
      tab_.alloc(std::max<size_t>(tab_host_.size(), 2 * tab_.n));  // all points are uploaded below
      graph_dirty_ = true;  // captured launches hold the old array
    }
    FMD_CUDA(cudaMemcpyAsync(tab_.p, tab_host_.data(), tab_host_.size() * sizeof(float2), cudaMemcpyHostToDevice, st_));
    FMD_CUDA(cudaStreamSynchronize(st_));
  }
  FMD_CUDA(cudaMemsetAsync(acf_.p + (size_t)r * kAcfWords, 0, kAcfWords * sizeof(double), st_));
  // Topology CSR by atom id.
  {
    const int n = t.natoms;
    std::vector<int32_t> boff(R.slot_cap, 0), aoff(R.slot_cap, 0);
    for (int b = 0; b < t.nbonds(); ++b) {
      boff[t.bonds[2 * b] + 1]++;
      boff[t.bonds[2 * b + 1] + 1]++;
    }
    for (int a = 0; a < t.nangles(); ++a)
      for (int k = 0; k < 3; ++k) aoff[t.angles[3 * a + k] + 1]++;
    for (int i = 0; i < n; ++i) {
      if (boff[i + 1] > kMaxBondsPerAtom || aoff[i + 1] > kMaxAnglesPerAtom) {
        throw Error(FMD_ERR_CONFIG, "an atom has more than 4 bonds or 8 angles (mixed-form limit)");
      }
    }
    for (int i = 0; i < n; ++i) {
      boff[i + 1] += boff[i];
      aoff[i + 1] += aoff[i];
    }
    std::vector<int2> be(std::max(1, 2 * t.nbonds()));
    std::vector<int4> ae(std::max(1, 3 * t.nangles()));
    std::vector<int32_t> fb(boff.begin(), boff.begin() + n), fa(aoff.begin(), aoff.begin() + n);
    for (int b = 0; b < t.nbonds(); ++b) {
      const int i = t.bonds[2 * b], j = t.bonds[2 * b + 1], ty = t.bond_type[b];
      be[fb[i]++] = make_int2(j, ty | (1 << 8));
      be[fb[j]++] = make_int2(i, ty);
    }
    for (int a = 0; a < t.nangles(); ++a) {
      const int i = t.angles[3 * a], j = t.angles[3 * a + 1], k = t.angles[3 * a + 2], ty = t.angle_type[a];
      ae[fa[i]++] = make_int4(i, j, k, ty | (0 << 8));
      ae[fa[j]++] = make_int4(i, j, k, ty | (1 << 8));
      ae[fa[k]++] = make_int4(i, j, k, ty | (2 << 8));
    }
    for (int i = n + 1; i < R.slot_cap; ++i) {
      boff[i] = boff[n];
      aoff[i] = aoff[n];
    }
    FMD_CUDA(cudaMemcpyAsync(boff_.p + R.slot_base, boff.data(), R.slot_cap * sizeof(int32_t), cudaMemcpyHostToDevice, st_));
    FMD_CUDA(cudaMemcpyAsync(aoff_.p + R.slot_base, aoff.data(), R.slot_cap * sizeof(int32_t), cudaMemcpyHostToDevice, st_));
    if (t.nbonds())
      FMD_CUDA(cudaMemcpyAsync(bent_.p + R.bond_base, be.data(), 2 * t.nbonds() * sizeof(int2), cudaMemcpyHostToDevice, st_));
    if (t.nangles())
      FMD_CUDA(cudaMemcpyAsync(aent_.p + R.angle_base, ae.data(), 3 * t.nangles() * sizeof(int4), cudaMemcpyHostToDevice, st_));
  }
  for (int c = 0; c < p.nchunks; ++c)
    h_chunk_rep_[ch + c] = make_int4(r, (int)(ch * kChunk) + c * kChunk, std::max(0, std::min(kChunk, t.natoms - c * kChunk)), c);
  FMD_CUDA(cudaMemcpyAsync(chunk_rep_.p + ch, h_chunk_rep_.data() + ch, p.nchunks * sizeof(int4), cudaMemcpyHostToDevice, st_));
  FMD_CUDA(cudaMemsetAsync(cell_cnt_.p + ce, 0, p.ncell * sizeof(int32_t), st_));
  hw_nreps_ = std::max(hw_nreps_, r + 1);
  hw_cells_ = std::max<int>(hw_cells_, (int)p.ncell);
  hw_home_ = std::max<int>(hw_home_, p.G_alloc * p.G_alloc * p.G_alloc);
  // Other replicas must not advance while this one is being set up.
  download_reps_keep(r);
  upload_atoms(r, t.xyz.data(), t.vel.data(), t.image.data());
  if (pushoff && pushoff->pushoff_steps > 0) {
    // Capped-force push-off runs batched with every other replica admitted
    // since the last run() (finish_pushoffs); forces are capped from setup on.
    Rep& P = h_reps_[r];
    P.mode = kModePushoff;
    P.fcap = pushoff->pushoff_fcap > 0 ? pushoff->pushoff_fcap : 50.0;
    P.push_dt = pushoff->pushoff_dt > 0 ? pushoff->pushoff_dt : 0.005;
    info_[r].pending_pushoff = pushoff->pushoff_steps;
  }
  setup({r});
  return r;
}

void Batch::finish_pushoffs() {
  std::vector<int> pend;
  int64_t steps = 0;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && info_[r].pending_pushoff > 0) {
      pend.push_back(r);
      steps = std::max(steps, info_[r].pending_pushoff);
    }
  if (pend.empty()) return;
  download_reps();
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used) h_reps_[r].stop_step = h_reps_[r].step;
  for (int r : pend) {
    h_reps_[r].step = 0;
    h_reps_[r].stop_step = info_[r].pending_pushoff;
  }
  upload_reps();
  int64_t direct = steps;
  if (graph_steps_ > 0 && steps >= graph_steps_) {
    ensure_graph();
    for (int64_t k = 0; k < steps / graph_steps_; ++k) FMD_CUDA(cudaGraphLaunch(graph_exec_, st_));
    direct = steps % graph_steps_;
  }
  const Dev d = dev();
  for (int64_t k = 0; k < direct; ++k) launch_step(d, shape(), &host_mode_, st_);
  FMD_CUDA_LAUNCH();
  FMD_CUDA(cudaStreamSynchronize(st_));
  download_reps();
  complete_pushoffs(pend);
}

// Concurrent push-offs (run() advanced them beside the running replicas):
// those that reached their length start their run.
void Batch::complete_done_pushoffs() {
  std::vector<int> done;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && info_[r].pending_pushoff > 0 && h_reps_[r].step >= info_[r].pending_pushoff)
      done.push_back(r);
  complete_pushoffs(done);
}

// Replicas whose push-off is done start their run: run mode, step 0, fresh
// thermostat / barostat state, a rebuild and first forces.
void Batch::complete_pushoffs(const std::vector<int>& pend) {
  if (pend.empty()) return;
  for (int r : pend) {
    info_[r].pending_pushoff = 0;
    Rep& R3 = h_reps_[r];
    R3.mode = kModeRun;
    R3.fcap = 0;
    R3.step = 0;
    R3.stop_step = 0;
    std::memset(&R3.nh, 0, sizeof(R3.nh));
    R3.nh.scale = 1.0;
    R3.nh.bscale = 1.0;
    R3.nh.exp_vW = 1.0;
    R3.nh.L = R3.L;
    R3.nh.inv_L = 1.0 / R3.L;
    R3.nh.V = R3.L * R3.L * R3.L;
    R3.nh.carry_dd = R3.chain_carry;
    R3.pending_scale = 1.0;
    R3.rebuilds = 0;
  }
  upload_reps();
  setup(pend);
}

// Refresh the host mirror of every replica except r (whose record the host
// has just written) from the device.
void Batch::download_reps_keep(int r) {
  const Rep keep = h_reps_[r];
  download_reps();
  h_reps_[r] = keep;
}

void Batch::freeze_others(int r) {
  for (int k = 0; k < max_reps_; ++k)
    if (k != r && info_[k].used) h_reps_[k].stop_step = h_reps_[k].step;
}

// Rebuild + forces + KE reduction without integrating (main.cu:313-390), for
// the listed replicas; the others are left untouched.
void Batch::setup(const std::vector<int>& rs) {
  for (int k = 0; k < max_reps_; ++k)
    if (info_[k].used) h_reps_[k].stop_step = h_reps_[k].step;
  for (int r : rs) {
    Rep& R = h_reps_[r];
    R.adv = 1;
    R.rebuild_now = 1;
    R.since = 0;
    R.L_list = R.L;
    R.list_scale = 1.0;
    R.L_filter = R.L;
    R.filter_scale = 1.0;
    R.maxdisp_bits = 0;
    R.disp_acc = 0.f;
    R.force_ev = 1;
  }
  upload_reps();
  // the rebuild work list holds exactly these replicas
  write_rebuild_list(rs);
  const Dev d = dev();
  launch_rebuild(d, nreps_launch(), nbr_variant_, st_);
  FMD_CUDA_LAUNCH();
  launch_forces_only(d, nchunks_launch(), force_variant_, shape().has_table != 0, st_);
  FMD_CUDA_LAUNCH();
  launch_reduce_only(d, nchunks_launch(), nreps_launch(), st_, 0);
  FMD_CUDA_LAUNCH();
  download_reps();
  for (int r : rs) check_status(r, true);
}

void Batch::check_status(int r, bool throw_on_fault) {
  const Rep& R = h_reps_[r];
  if (R.status == 0) return;
  if (!throw_on_fault) return;
  if (R.status & kStatusOverflow) throw Error(FMD_ERR_OVERFLOW, "neighbor list overflow");
  if (R.status & kStatusCellCapacity) throw Error(FMD_ERR_OVERFLOW, "cell grid capacity exceeded");
  if (R.status & kStatusNonFinite) throw Error(FMD_ERR_FAULT, "non-finite state");
  if (R.status & kStatusFeneStretch) throw Error(FMD_ERR_FAULT, "FENE bond stretched to R0");
  if (R.status & kStatusStaleScalars) throw Error(FMD_ERR_FAULT, "pre-force step without its step scalars");
  throw Error(FMD_ERR_FAULT, "replica fault");
}

void Batch::advance_direct(int64_t nsteps) {
  const Dev d = dev();
    for (int64_t k = 0; k < nsteps; ++k) launch_step(d, shape(), &host_mode_, st_);
  FMD_CUDA_LAUNCH();
  FMD_CUDA(cudaStreamSynchronize(st_));
}

static bool same_shape(const StepShape& a, const StepShape& b) {
  return a.nchunks == b.nchunks && a.nreps == b.nreps && a.max_cells == b.max_cells && a.max_home == b.max_home &&
         a.force_variant == b.force_variant && a.nbr_variant == b.nbr_variant && a.has_table == b.has_table;
}

void Batch::ensure_graph() {
  const StepShape want = shape();
  if (!graph_dirty_ && graph_exec_ && same_shape(want, graph_shape_)) return;
  if (graph_exec_) {
    cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
  }
  const Dev d = dev();
    cudaGraph_t g;
  FMD_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  try {
    for (int k = 0; k < graph_steps_; ++k) capture_step(d, want, st_, side_, side_hi_, branch_);
  } catch (...) {
    cudaGraph_t partial = nullptr;
    cudaStreamEndCapture(st_, &partial);
    if (partial) cudaGraphDestroy(partial);
    throw;
  }
  FMD_CUDA(cudaStreamEndCapture(st_, &g));
  // per-node priorities: the rebuild branch's kernels are dispatched ahead of
  // the force kernels that run beside them
  FMD_CUDA(cudaGraphInstantiate(&graph_exec_, g, cudaGraphInstantiateFlagUseNodePriority));
  cudaGraphDestroy(g);
  graph_dirty_ = false;
  graph_shape_ = want;
  ++graph_captures_;
}

void Batch::run(int64_t nsteps, bool respect_nsteps) {
  if (!concurrent_pushoff_) finish_pushoffs();
  if (nsteps <= 0) return;
  download_reps();
  int64_t need = 0;
  for (int r = 0; r < max_reps_; ++r) {
    if (!info_[r].used) continue;
    Rep& R = h_reps_[r];
    if (!R.active) {
      R.stop_step = R.step;
      continue;
    }
    int64_t stop = R.step + nsteps;
    if (info_[r].pending_pushoff > 0)  // concurrent push-off: its own length
      stop = std::min<int64_t>(stop, info_[r].pending_pushoff);
    else if (respect_nsteps && R.nsteps > 0)
      stop = std::min<int64_t>(stop, R.nsteps);
    R.stop_step = stop;
    need = std::max<int64_t>(need, stop - R.step);
  }
  if (need == 0) {
    if (concurrent_pushoff_) complete_done_pushoffs();
    return;
  }
  upload_reps();
  if (graph_steps_ > 0 && need >= graph_steps_) {
    ensure_graph();
    const int64_t reps = need / graph_steps_;
    for (int64_t k = 0; k < reps; ++k) FMD_CUDA(cudaGraphLaunch(graph_exec_, st_));
    need -= reps * graph_steps_;
  }
  if (need > 0) {
    const Dev d = dev();
    for (int64_t k = 0; k < need; ++k) launch_step(d, shape(), &host_mode_, st_);
    FMD_CUDA_LAUNCH();
  }
  FMD_CUDA(cudaStreamSynchronize(st_));
  download_reps();
  if (concurrent_pushoff_) complete_done_pushoffs();
  // A faulted replica stops; the others continue.
  bool changed = false;
  for (int r = 0; r < max_reps_; ++r) {
    if (!info_[r].used) continue;
    Rep& R = h_reps_[r];
    if (R.status != 0 && R.active) {
      R.active = 0;
      changed = true;
    }
  }
  if (changed) upload_reps();
}

void Batch::retire(int r) {
  if (r < 0 || r >= max_reps_ || !info_[r].used) throw Error(FMD_ERR_ARG, "no such replica");
  download_reps();
  ReplicaInfo& I = info_[r];
  Rep& R = h_reps_[r];
  for (int c = 0; c < R.nchunks; ++c) h_chunk_rep_[R.chunk_base + c] = make_int4(-1, 0, 0, 0);
  FMD_CUDA(cudaMemcpyAsync(chunk_rep_.p + R.chunk_base, h_chunk_rep_.data() + R.chunk_base, R.nchunks * sizeof(int4),
                           cudaMemcpyHostToDevice, st_));
  slot_alloc_.release(I.seg_chunk);
  cell_alloc_.release(I.seg_cell);
  nbr_alloc_.release(I.seg_nbr);
  bond_alloc_.release(I.seg_bond);
  angle_alloc_.release(I.seg_angle);
  bytes_in_use_ -= I.bytes;
  R = Rep{};
  I = ReplicaInfo{};
  upload_reps();
  FMD_CUDA(cudaStreamSynchronize(st_));
}

void Batch::mark(int which) {
  if (which < 0 || which > 1) throw Error(FMD_ERR_ARG, "event index must be 0 or 1");
  if (!ev_[which]) FMD_CUDA(cudaEventCreate(&ev_[which]));
  FMD_CUDA(cudaEventRecord(ev_[which], st_));
}

double Batch::elapsed_ms() {
  if (!ev_[0] || !ev_[1]) throw Error(FMD_ERR_STATE, "both events must be recorded first");
  FMD_CUDA(cudaEventSynchronize(ev_[1]));
  float ms = 0;
  FMD_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
  return ms;
}

// Device time per launch of the force kernel on the current state (the
// evaluation is idempotent); variant < 0: the batch's current variant.  Only
// the kernel flavour the replicas need (with or without energies) is timed.
double Batch::time_force(int iters, int variant, bool steady) {
  if (variant < 0) variant = force_variant_;
  download_reps();
  // mark every replica as advancing for the force kernel only
  std::vector<Rep> saved = h_reps_;
  bool any_ev = false, any_plain = false;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && h_reps_[r].active) {
      h_reps_[r].adv = 1;
      if (steady) {
        h_reps_[r].force_ev = 0;
        h_reps_[r].thermo_freq = 0;
        h_reps_[r].stress_freq = 0;
      }
      (need_ev(h_reps_[r]) ? any_ev : any_plain) = true;
    }
  upload_reps();
  const Dev d = dev();
  const int nc = nchunks_launch();
  auto once = [&] {
    if (any_plain) launch_force(d, nc, false, variant, st_, false);
    if (any_ev) launch_force(d, nc, true, variant, st_, false);
  };
  once();  // warm
  FMD_CUDA_LAUNCH();
  mark(0);
  for (int k = 0; k < iters; ++k) once();
  FMD_CUDA_LAUNCH();
  mark(1);
  const double ms = elapsed_ms() / std::max(1, iters);
  h_reps_ = saved;
  upload_reps();
  FMD_CUDA(cudaStreamSynchronize(st_));
  return ms;
}

// Device time of a rebuild of every active replica with neighbor-list
// variant v.  A rebuild of an unchanged state reproduces it (same cells, same
// in-cell order, identity permutation); it resets the displacement reference.
double Batch::time_rebuild(int iters, int v) {
  download_reps();
  std::vector<int> rs;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && h_reps_[r].active) rs.push_back(r);
  if (rs.empty()) return 0.0;
  for (int r : rs) {
    h_reps_[r].rebuild_now = 1;  // the rebuild kernels act on replicas marked so
    h_reps_[r].maxdisp_bits = 0;
    h_reps_[r].disp_acc = 0.f;
  }
  upload_reps();
  const Dev d = dev();
  auto once = [&] {
    write_rebuild_list(rs);
    launch_rebuild(d, nreps_launch(), v, st_);
  };
  once();
  FMD_CUDA_LAUNCH();
  mark(0);
  for (int k = 0; k < iters; ++k) once();
  FMD_CUDA_LAUNCH();
  mark(1);
  const double ms = elapsed_ms() / std::max(1, iters);
  FMD_CUDA(cudaStreamSynchronize(st_));
  return ms;
}

// Time every force-kernel variant on the live state and keep the fastest,
// then every neighbor-list variant on a full rebuild (the step graph is
// re-captured with the choices).
int Batch::autotune(int iters, double* ms_out, int cap) {
  int nb = 0;
  double nb_ms = 0;
  for (int v = 0; v < kNbrVariants; ++v) {
    const double ms = time_rebuild(std::max(1, iters / 5), v);
    nbr_ms_[v] = ms;
    if (v == 0 || ms < nb_ms) {
      nb = v;
      nb_ms = ms;
    }
  }
  if (nb != nbr_variant_) graph_dirty_ = true;
  nbr_variant_ = nb;
  int best = 0;
  double best_ms = 0;
  for (int v = 0; v < kForceVariants; ++v) {
    const double ms = time_force(iters, v, true);
    if (ms_out && v < cap) ms_out[v] = ms;
    if (v == 0 || ms < best_ms) {
      best = v;
      best_ms = ms;
    }
  }
  if (best != force_variant_) graph_dirty_ = true;
  force_variant_ = best;
  // Rebuild cadence: the skin/2 displacement trigger alone keeps every pair
  // within rc listed, so a forced cadence (the reference's 20 steps) only
  // adds rebuilds; it is lifted for the active replicas (set_max_between
  // restores one).
  download_reps();
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && h_reps_[r].active) h_reps_[r].max_between = kNoForcedRebuild;
  upload_reps();
  FMD_CUDA(cudaStreamSynchronize(st_));
  // List buffer: where a replica keeps a pruned list, the force kernels walk
  // that list whatever the Verlet list's margin, so the margin is widened to
  // the cell edge (the widest the cell grid allows unchanged): the list
  // build, per atom the costliest work of a step, then runs less often.
  for (int r = 0; r < max_reps_; ++r) {
    if (!info_[r].used || !h_reps_[r].active) continue;
    const Rep& R = h_reps_[r];
    if (!(R.prune_delta > 0.f) || R.G < 3) continue;
    const double wide = R.L / (1.0002 * R.G) - R.rc;
    const double rcs = R.rc + wide;
    const double expect = R.natoms / (R.L * R.L * R.L) * (4.0 / 3.0) * 3.14159265358979323846 * rcs * rcs * rcs;
    if (wide > R.skin + 0.02 && 1.3 * expect + 16.0 <= R.M) set_list_buffer(r, wide);
  }
  return best;
}

void Batch::set_variants(int fv, int nv) {
  if (fv >= kForceVariants || nv >= kNbrVariants) throw Error(FMD_ERR_ARG, "no such kernel variant");
  if (fv >= 0 && fv != force_variant_) {
    force_variant_ = fv;
    graph_dirty_ = true;
  }
  if (nv >= 0 && nv != nbr_variant_) {
    nbr_variant_ = nv;
    graph_dirty_ = true;
  }
}

void Batch::last_forces(int r, double* f) {
  const Rep& R = rep(r);
  const int n = R.natoms;
  std::vector<float4> hf(n);
  std::vector<int4> hi(n);
  FMD_CUDA(cudaMemcpyAsync(hf.data(), force_.p + R.slot_base, n * sizeof(float4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaMemcpyAsync(hi.data(), img_.p + R.slot_base, n * sizeof(int4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
  for (int s = 0; s < n; ++s) {
    const int id = hi[s].w;
    f[3 * id] = hf[s].x;
    f[3 * id + 1] = hf[s].y;
    f[3 * id + 2] = hf[s].z;
  }
}

void Batch::list_stats(int64_t* entries, int32_t* max_per_atom) {
  int64_t tot = 0;
  int32_t mx = 0;
  for (int r = 0; r < max_reps_; ++r) {
    if (!info_[r].used || !h_reps_[r].active) continue;
    const Rep& R = h_reps_[r];
    std::vector<int32_t> c(R.natoms);
    // the list the force kernel walks: the pruned one where the replica keeps it
    const int32_t* src = (R.prune_delta > 0.f ? pcnt_.p : ncnt_.p) + R.slot_base;
    FMD_CUDA(cudaMemcpy(c.data(), src, R.natoms * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (int32_t v : c) {
      tot += v;
      mx = std::max(mx, v);
    }
  }
  if (entries) *entries = tot;
  if (max_per_atom) *max_per_atom = mx;
}

// Turn a replica's pruned list on (margin delta beyond rc) or off (delta <=
// 0).  Turning it on filters the list at once.
void Batch::set_list_prune(int r, double delta) {
  download_reps();
  Rep& R = h_reps_[r];
  const bool on = delta > 0.0;
  R.prune_delta = on ? (float)delta : 0.f;
  if (on) {
    // a filter now: the displacement since the last reference joins the
    // accumulated bound and the current positions become the reference
    R.disp_acc += std::sqrt(uint_as_float_host(R.maxdisp_bits));
    R.maxdisp_bits = 0;
    R.L_filter = R.L;
    R.filter_scale = 1.0;
    R.rebuild_now = 2;
    upload_reps();
    write_rebuild_list(std::vector<int>{r}, 0);
    launch_prune_only(dev(), st_);
    FMD_CUDA_LAUNCH();
    R.rebuild_now = 0;
  }
  upload_reps();
  FMD_CUDA(cudaStreamSynchronize(st_));
}

// The Verlet list's margin beyond rc (the run.conf skin until changed): the
// list holds the pairs within rc + skin and a rebuild follows a displacement
// of skin / 2.  Changing it rebuilds the replica's list at once.
void Batch::set_list_buffer(int r, double skin) {
  download_reps();
  Rep& R = h_reps_[r];
  if (!(skin > 0.0) || !std::isfinite(skin)) throw Error(FMD_ERR_ARG, "list buffer must be positive");
  const double rcs = R.rc + skin;
  const double rho = R.natoms / (R.L * R.L * R.L);
  const double expect = rho * (4.0 / 3.0) * 3.14159265358979323846 * rcs * rcs * rcs;
  if (1.3 * expect + 16.0 > R.M) throw Error(FMD_ERR_ARG, "list buffer too wide for the replica's list capacity");
  R.skin = skin;
  R.rebuild_now = 1;
  R.maxdisp_bits = 0;
  R.disp_acc = 0.f;
  upload_reps();
  write_rebuild_list(std::vector<int>{r});
  launch_rebuild(dev(), nreps_launch(), nbr_variant_, st_);
  FMD_CUDA_LAUNCH();
  R.rebuild_now = 0;
  upload_reps();
  FMD_CUDA(cudaStreamSynchronize(st_));
}

void Batch::set_max_between(int r, int k) {
  download_reps();
  h_reps_[r].max_between = k > 0 ? k : kNoForcedRebuild;
  upload_reps();
  FMD_CUDA(cudaStreamSynchronize(st_));
}

const Rep& Batch::rep(int r) const {
  if (r < 0 || r >= max_reps_ || !info_[r].used) throw Error(FMD_ERR_ARG, "no such replica");
  return h_reps_[r];
}

void Batch::get_state(int r, double* xyz, double* vel, int32_t* image) { read_state(r, xyz, vel, image, true); }

void Batch::pack_frame(int r, float* d_xyz, float* h_xyz, cudaEvent_t ready) {
  const Rep& R = rep(r);
  launch_pack_frame(dev(), r, R.natoms, d_xyz, st_);
  FMD_CUDA_LAUNCH();
  FMD_CUDA(cudaMemcpyAsync(h_xyz, d_xyz, (size_t)R.natoms * 3 * sizeof(float), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaEventRecord(ready, st_));
}

void Batch::force_frame(int r, double* xyz, double* box) {
  read_state(r, xyz, nullptr, nullptr, false);
  if (box) *box = rep(r).Lpos;
}

void Batch::read_state(int r, double* xyz, double* vel, int32_t* image, bool rewrap) {
  const Rep& R = rep(r);
  const int n = R.natoms;
  std::vector<float4> hp(n), hv(n);
  std::vector<int4> hi(n);
  FMD_CUDA(cudaMemcpyAsync(hp.data(), pos_.p + R.slot_base, n * sizeof(float4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaMemcpyAsync(hv.data(), vel_.p + R.slot_base, n * sizeof(float4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaMemcpyAsync(hi.data(), img_.p + R.slot_base, n * sizeof(int4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
  // The reference wraps positions in the box of the last pre-force update
  // (Lpos); an NPT barostat has changed L since, and positions are reported
  // re-wrapped into the current box L (two wraps, the first one in Lpos).
  const double Lp = R.Lpos, L = R.L, h = R.h;
  for (int s = 0; s < n; ++s) {
    const int id = hi[s].w;
    const uint32_t u = w_bits(hp[s].w);
    const int c[3] = {w_cx(u), w_cy(u), w_cz(u)};
    const float o[3] = {hp[s].x, hp[s].y, hp[s].z};
    const int im[3] = {hi[s].x, hi[s].y, hi[s].z};
    for (int a = 0; a < 3; ++a) {
      double x = (double)c[a] * h + (double)o[a];
      int ia = im[a];
      double fl = std::floor(x / Lp);
      x -= fl * Lp;
      ia += (int)fl;
      if (rewrap) {
        fl = std::floor(x / L);
        x -= fl * L;
        ia += (int)fl;
      }
      if (xyz) xyz[3 * id + a] = x;
      if (image) image[3 * id + a] = ia;
    }
    if (vel) {
      vel[3 * id] = (double)hv[s].x * R.pending_scale;
      vel[3 * id + 1] = (double)hv[s].y * R.pending_scale;
      vel[3 * id + 2] = (double)hv[s].z * R.pending_scale;
    }
  }
}

// The rebuild work list holds exactly these replicas (a host-driven rebuild).
void Batch::write_rebuild_list(const std::vector<int>& rs, int rebuilds) {
  wl_.assign(kRbHead + rs.size(), 0);
  wl_[kRbCount] = (int)rs.size();
  wl_[kRbRebuilds] = rebuilds < 0 ? (int)rs.size() : rebuilds;
  wl_[kRbMode] = kRbList;
  std::copy(rs.begin(), rs.end(), wl_.begin() + kRbHead);
  FMD_CUDA(cudaMemcpyAsync(rb_.p, wl_.data(), wl_.size() * sizeof(int), cudaMemcpyHostToDevice, st_));
}

void Batch::launch_counts(int64_t* counts, int n) {
  unsigned long long h[kKernelKinds];
  FMD_CUDA(cudaMemcpyAsync(h, kcount_.p, sizeof(h), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
  for (int k = 0; k < n && k < kKernelKinds; ++k) counts[k] = (int64_t)h[k];
}

void Batch::write_restart(int r, const std::string& path) {
  Topology t = info_[r].topo;
  StateFile st;
  checkpoint(r, t, st);
  write_lammps_data(path, t, rep(r).step);
  write_state_file(state_path(path), st);
}

namespace {
// Sidecar values of a replica's dynamic state (what a data file lacks).
void put_nh(StateFile& s, const NHScalars& nh) {
  s.put("nh_xi", std::vector<double>(nh.xi, nh.xi + 10));
  s.put("nh_vxi", std::vector<double>(nh.vxi, nh.vxi + 10));
  s.put("nh_scalars", {nh.eps, nh.veps, nh.carry, nh.scale, nh.L, nh.inv_L, nh.V, nh.bscale, nh.exp_vW, nh.vWdt,
                       nh.fpos, nh.ke_raw, nh.vir_tr});
  s.put("nh_dd", std::vector<double>(nh.dd, nh.dd + 10));
}
void get_nh(const StateFile& s, NHScalars& nh) {
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
}
}  // namespace

void Batch::checkpoint(int r, Topology& t, StateFile& s) {
  rep(r);
  const size_t n = (size_t)h_reps_[r].natoms;
  t.xyz.resize(3 * n);
  t.vel.resize(3 * n);
  t.image.resize(3 * n);
  get_state(r, t.xyz.data(), t.vel.data(), t.image.data());
  download_reps();
  const Rep& R = h_reps_[r];
  t.box_L = R.L;
  s.put("form", {1.0});
  s.put("natoms", {(double)R.natoms});
  s.put("ensemble", {(double)R.ensemble});
  s.put("step", {(double)R.step});
  s.put("box_L", {R.L});
  s.put("V0", {R.V0});
  s.put("rebuilds", {(double)R.rebuilds});
  s.put("list_buffer", {R.skin});
  s.put("rebuild_cadence", {(double)R.max_between});
  s.put("prune_delta", {(double)R.prune_delta});
  put_nh(s, R.nh);
  // continue from exactly what a resumed run starts from
  restore(r, t, s);
}

void Batch::restore(int r, const Topology& t, const StateFile& s) {
  rep(r);
  download_reps();
  Rep& R = h_reps_[r];
  if ((int)s.get1("natoms") != R.natoms) throw Error(FMD_ERR_IO, "restart state is for another atom count");
  if ((int)s.get1("ensemble") != R.ensemble) throw Error(FMD_ERR_IO, "restart state is for another ensemble");
  R.step = (int64_t)s.get1("step");
  R.L = s.get1("box_L");
  R.V0 = s.get1("V0");
  if (s.has("rebuilds")) R.rebuilds = (int64_t)s.get1("rebuilds");
  if (s.has("list_buffer")) R.skin = s.get1("list_buffer");
  if (s.has("rebuild_cadence")) R.max_between = (int32_t)s.get1("rebuild_cadence");
  if (s.has("prune_delta")) R.prune_delta = (float)s.get1("prune_delta");
  get_nh(s, R.nh);
  // the cell grid of the box, as a fresh replica derives it
  int G = (int)std::floor(R.L / ((R.rc + R.skin) * 1.0001));
  R.G = std::max(1, std::min(G, R.G_alloc));
  upload_reps();
  set_state(r, t.xyz.data(), t.vel.data(), t.image.data());
}

void Batch::set_state(int r, const double* xyz, const double* vel, const int32_t* image) {
  const Rep& R0 = rep(r);
  const int n = R0.natoms;
  std::vector<double> x(3 * n), v(3 * n);
  std::vector<int32_t> im(3 * n);
  get_state(r, x.data(), v.data(), im.data());
  if (xyz) std::memcpy(x.data(), xyz, 3 * n * sizeof(double));
  if (vel) std::memcpy(v.data(), vel, 3 * n * sizeof(double));
  if (image) std::memcpy(im.data(), image, 3 * n * sizeof(int32_t));
  else if (xyz) std::fill(im.begin(), im.end(), 0);
  download_reps();
  Rep& R = h_reps_[r];
  R.pending_scale = 1.0;
  R.defer = 0;
  R.Lpos = R.L;
  R.h = (float)(R.L / R.G);
  upload_atoms(r, x.data(), v.data(), im.data());
  setup({r});
}

// Energies and virial of the current state for replica r: steps between
// thermo steps skip them, so a readout re-evaluates the forces (same
// positions, same list, same result) with energies on.
// Energies and virial of the current state of replica r, re-evaluated when
// the last step did not compute them.  Every other running replica whose
// energies are stale is re-evaluated in the same pass: reading the thermo
// rows of a whole batch after a run costs one force pass, not one per
// replica (the forces are bit-identical to the step's, so this perturbs no
// trajectory).
void Batch::ensure_ev(int r) {
  rep(r);
  if (h_reps_[r].ev_step == h_reps_[r].step) return;
  for (int k = 0; k < max_reps_; ++k)
    if (info_[k].used) h_reps_[k].stop_step = h_reps_[k].step;
  for (int k = 0; k < max_reps_; ++k) {
    Rep& K = h_reps_[k];
    const bool stale = info_[k].used && K.active && K.mode == kModeRun && K.ev_step != K.step;
    if (k == r || stale) {
      K.adv = 1;
      K.force_ev = 1;
      K.rebuild_now = 0;
    }
  }
  upload_reps();
  const Dev d = dev();
  launch_forces_only(d, nchunks_launch(), force_variant_, shape().has_table != 0, st_);
  FMD_CUDA_LAUNCH();
  launch_reduce_only(d, nchunks_launch(), nreps_launch(), st_, 2);
  FMD_CUDA_LAUNCH();
  download_reps();
}

void Batch::forces(int r, double* f, double* pe, double* vir) {
  ensure_ev(r);
  const Rep& R = rep(r);
  const int n = R.natoms;
  std::vector<float4> hf(n);
  std::vector<int4> hi(n);
  FMD_CUDA(cudaMemcpyAsync(hf.data(), force_.p + R.slot_base, n * sizeof(float4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaMemcpyAsync(hi.data(), img_.p + R.slot_base, n * sizeof(int4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
  for (int s = 0; s < n; ++s) {
    const int id = hi[s].w;
    if (f) {
      f[3 * id] = hf[s].x;
      f[3 * id + 1] = hf[s].y;
      f[3 * id + 2] = hf[s].z;
    }
    if (pe) pe[id] = hf[s].w;
  }
  if (vir) std::memcpy(vir, R.vir, 6 * sizeof(double));
}

void Batch::thermo(int r, fmd_thermo_row* row) {
  ensure_ev(r);
  const Rep& R = rep(r);
  const int n = R.natoms;
  const double s2 = R.pending_scale * R.pending_scale;
  double k[6];
  for (int c = 0; c < 6; ++c) k[c] = R.ke[c] * s2;
  const double ke = 0.5 * (k[0] + k[3] + k[5]);
  row->step = R.step;
  row->ke = ke / n;
  row->pe = R.pe / n;
  row->temp = 2.0 * row->ke / 3.0;
  const double V = R.L * R.L * R.L;
  for (int c = 0; c < 6; ++c) row->stress[c] = (k[c] + R.vir[c]) / V;
  row->box_L = R.L;
  double e = ke + R.pe;
  if (R.ensemble != FMD_LANGEVIN) {
    const double frac = (double)(R.step - 1) / (double)(R.nsteps > 0 ? R.nsteps : 1);
    const double kT = R.T0 + (R.T1 - R.T0) * frac;
    const double Nf = 3.0 * n;
    e += 0.5 * R.Q1 * R.nh.vxi[0] * R.nh.vxi[0] + Nf * kT * R.nh.xi[0];
    for (int q = 1; q < R.chain_M; ++q) e += 0.5 * R.Qr * R.nh.vxi[q] * R.nh.vxi[q] + kT * R.nh.xi[q];
    if (R.ensemble == FMD_NPT_NH) {
      const double Pt = R.P0 + (R.P1 - R.P0) * frac;
      e += R.nh.veps * R.nh.veps / (2.0 * R.W) + Pt * V;
    }
  }
  row->conserved = e / n;
}

// Rows of the stress autocorrelation in the order of the reference's output
// file (main.cu:758-783): per level, per lag with samples, the lag in steps
// stress_freq * kAcfPoints^level * (lag + 1), the six averages and the count.
void Batch::stress_acf(int r, std::vector<int64_t>& lag, std::vector<double>& val, std::vector<int64_t>& cnt) {
  const Rep& R = rep(r);
  if (R.stress_freq <= 0) throw Error(FMD_ERR_ARG, "run.conf has no 'stress' output for this replica");
  std::vector<double> st(kAcfWords);
  FMD_CUDA(cudaMemcpyAsync(st.data(), acf_.p + (size_t)r * kAcfWords, kAcfWords * sizeof(double),
                           cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
  lag.clear();
  val.clear();
  cnt.clear();
  int64_t lag_step = R.stress_freq;
  for (int level = 0; level < kAcfLevels; ++level) {
    for (int k = 0; k < kAcfPoints; ++k) {
      const double n = st[kAcfCnt + level * kAcfPoints + k];
      if (n == 0.0) continue;
      lag.push_back(lag_step * (k + 1));
      for (int c = 0; c < kAcfComps; ++c) val.push_back(st[kAcfCorr + (level * kAcfPoints + k) * kAcfComps + c] / n);
      cnt.push_back((int64_t)n);
    }
    lag_step *= kAcfPoints;
  }
}

void Batch::write_stress_acf(int r, const std::string& path) {
  std::vector<int64_t> lag, cnt;
  std::vector<double> val;
  stress_acf(r, lag, val, cnt);
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw Error(FMD_ERR_IO, "cannot open " + path);
  std::fprintf(f, "# lag_steps  C_xx  C_xy  C_xz  C_yy  C_yz  C_zz  count\n");
  for (size_t i = 0; i < lag.size(); ++i) {
    std::fprintf(f, "%lld", (long long)lag[i]);
    for (int c = 0; c < kAcfComps; ++c) std::fprintf(f, " %.8e", val[i * kAcfComps + c]);
    std::fprintf(f, " %lld\n", (long long)cnt[i]);
  }
  std::fclose(f);
}

double Batch::rg(int r) {
  const Rep& R = rep(r);
  const int n = R.natoms;
  std::vector<double> x(3 * n);
  std::vector<int32_t> im(3 * n);
  // The reference unwraps the stored positions (wrapped in Lpos) with the
  // current box L (analysis/rg.cu).
  read_state(r, x.data(), nullptr, im.data(), false);
  const std::vector<int32_t>& mol = info_[r].mol;
  std::vector<int32_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return mol[a] < mol[b]; });
  double sum = 0;
  int nch = 0;
  const double L = R.L;
  for (int s = 0; s < n;) {
    int e = s;
    while (e < n && mol[order[e]] == mol[order[s]]) ++e;
    double com[3] = {0, 0, 0};
    for (int t = s; t < e; ++t)
      for (int a = 0; a < 3; ++a) com[a] += x[3 * order[t] + a] + im[3 * order[t] + a] * L;
    for (int a = 0; a < 3; ++a) com[a] /= (e - s);
    double rg2 = 0;
    for (int t = s; t < e; ++t)
      for (int a = 0; a < 3; ++a) {
        const double u = x[3 * order[t] + a] + im[3 * order[t] + a] * L - com[a];
        rg2 += u * u;
      }
    sum += std::sqrt(rg2 / (e - s));
    ++nch;
    s = e;
  }
  return nch ? sum / nch : 0.0;
}

int64_t Batch::pairs(int r, int32_t* pi, int32_t* pj, int64_t cap) {
  const Rep& R = rep(r);
  const int n = R.natoms;
  const int tiles = R.slot_cap / kTile;
  std::vector<uint32_t> nb((size_t)tiles * R.M * kTile);
  std::vector<int32_t> cnt(n);
  std::vector<int4> hi(n);
  FMD_CUDA(cudaMemcpyAsync(nb.data(), nbr_.p + R.nbr_base, nb.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaMemcpyAsync(cnt.data(), ncnt_.p + R.slot_base, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaMemcpyAsync(hi.data(), img_.p + R.slot_base, n * sizeof(int4), cudaMemcpyDeviceToHost, st_));
  FMD_CUDA(cudaStreamSynchronize(st_));
  int64_t m = 0;
  for (int s = 0; s < n; ++s)
    for (int k = 0; k < cnt[s]; ++k) {
      const uint32_t w = nb[((size_t)(s >> 5) * R.M + k) * kTile + (s & 31)];
      const int js = (int)(w & kIdxMask);
      const int a = hi[s].w, b = hi[js].w;
      if (a < b) {
        if (m < cap) {
          pi[m] = a;
          pj[m] = b;
        }
        ++m;
      }
    }
  return m;
}

void Batch::totals(int32_t* active, int64_t* atoms, int64_t* bytes) {
  int32_t a = 0;
  int64_t n = 0;
  for (int r = 0; r < max_reps_; ++r)
    if (info_[r].used && h_reps_[r].active) {
      ++a;
      n += h_reps_[r].natoms;
    }
  if (active) *active = a;
  if (atoms) *atoms = n;
  if (bytes) *bytes = bytes_in_use_;
}

// ------------------------------------------------------------- SimEngine
class MixedEngine final : public SimEngine {
 public:
  MixedEngine(const RunConfig& cfg, Topology t, const fmd_melt_spec* pushoff) {
    const ReplicaPlan p = plan_replica(cfg, t.natoms, t.box_L);
    BatchCaps c;
    c.slots = p.slot_cap;
    c.nbr = ((p.nbr_entries + 1023) / 1024) * 1024;
    c.cells = p.ncell;
    c.bonds = std::max<int64_t>(1, 2ll * t.nbonds());
    c.angles = std::max<int64_t>(1, 3ll * t.nangles());
    fmd_batch_opts o{};
    o.max_replicas = 1;
    o.hbm_budget_gb = 1e6;
    o.graph_steps = 20;
    b_.reset(new Batch(o, &c));
    nb_ = t.nbonds();
    na_ = t.nangles();
    r_ = b_->add(cfg, std::move(t), pushoff);
    b_->finish_pushoffs();
  }
  void step(int64_t n) override {
    b_->run(n, false);
    b_->check_status(r_, true);
  }
  void compute_forces(double* f, double* pe, double* vir) override { b_->forces(r_, f, pe, vir); }
  void get_state(double* x, double* v, int32_t* i) override { b_->get_state(r_, x, v, i); }
  void set_state(const double* x, const double* v, const int32_t* i) override { b_->set_state(r_, x, v, i); }
  void checkpoint(Topology& t, StateFile& s) override { b_->checkpoint(r_, t, s); }
  void restore(const Topology& t, const StateFile& s) override { b_->restore(r_, t, s); }
  void thermo(fmd_thermo_row* row) override { b_->thermo(r_, row); }
  double rg() override { return b_->rg(r_); }
  int64_t pairs(int32_t* pi, int32_t* pj, int64_t cap) override { return b_->pairs(r_, pi, pj, cap); }
  int32_t natoms() const override { return b_->rep(r_).natoms; }
  int32_t nbonds() const override { return nb_; }
  int32_t nangles() const override { return na_; }
  int64_t step_count() const override { return b_->rep(r_).step; }
  double box_L() override { return b_->rep(r_).L; }
  int64_t rebuilds() const override { return b_->rep(r_).rebuilds; }
  int32_t status_word() override { return b_->rep(r_).status; }
  int32_t max_neighbors() const override { return b_->rep(r_).M; }
  void stress_acf(std::vector<int64_t>& lag, std::vector<double>& val, std::vector<int64_t>& cnt) override {
    b_->stress_acf(r_, lag, val, cnt);
  }
  void write_stress_acf(const std::string& path) override { b_->write_stress_acf(r_, path); }
  void dump_frame(TrajWriter& w) override { w.write(*b_, r_); }

 private:
  std::unique_ptr<Batch> b_;
  int r_ = 0;
  int32_t nb_ = 0, na_ = 0;
};

}  // namespace mixed

std::unique_ptr<SimEngine> make_mixed_engine(const RunConfig& cfg, Topology topo, const fmd_melt_spec* pushoff) {
  return std::unique_ptr<SimEngine>(new mixed::MixedEngine(cfg, std::move(topo), pushoff));
}

}  // namespace fmd
