// Mixed-precision batched engine: kernels.
//
// One step over every replica of a batch (one block per 128-slot chunk for
// per-atom work; a chunk never straddles replicas):
//   k_pre        half kick / drift (Langevin BAOAB or Nose-Hoover NVT / MTK NPT)
//                on FP32 cell offsets with the replica's precomputed FP64 step
//                scalars; per-replica max displacement.
//   k_commit     one thread per replica: commits the step (chain / barostat
//                state, box), takes the rebuild decision (skin/2 displacement
//                or forced cadence) and appends to the rebuild work list; in a
//                CUDA graph it switches the conditional nodes below.
//   rebuild      [IF any replica rebuilds] work-list kernels over the flagged
//                replicas only: re-bin into cells, per-cell deterministic order,
//                permute state, per-slot bonded tables, Verlet lists.
//   k_force      [IF needed, with / without energies] LJ over the list +
//                FENE/WCA + harmonic angle gathered per atom (no atomics),
//                FP32 with compensated sums, FP64 block partials.
//   k_post       [IF needed] final half kick + FP64 KE-tensor partials, then
//   k_post_commit  one warp per replica reduces the partials in chunk order
//                and runs the post-force thermostat / barostat.  Langevin
//                steps inside a graph fold the final half kick into the next
//                k_pre instead (same operations, same order).
// Reference algorithm sources: integrate/langevin.cu:34-130,
// integrate/nose_hoover.cu:86-305, 606-898, force/lj.cu:21-65,
// force/fene.cu:18-73, force/angle.cu:17-80, neighbor/verlet_list.cu:108-335,
// neighbor/skin_trigger.cuh:6-33, analysis/thermo.cu:88-138.
#include <cuda_runtime.h>

#include "counter_rng.h"
#include "dev_common.cuh"
#include "mixed.cuh"
#include "nhc.h"

namespace fmd {
namespace mixed {

struct DExp {
  __device__ double operator()(double x) const { return exp(x); }
};
struct DCbrt {
  __device__ double operator()(double x) const { return cbrt(x); }
};
struct DSinh {
  __device__ double operator()(double x) const { return sinh(x); }
};

__device__ __forceinline__ double ramp(const Rep& R, int64_t step, double a, double b) {
  const double frac = (double)(step - 1) / (double)(R.nsteps > 0 ? R.nsteps : 1);
  return a + (b - a) * frac;
}

// Scalars of the step after R.step.  The single-thread commit kernels inline
// this into a local and store the result once (next_scalars): through a
// reference that may point into R (R.next), every store would order the
// later reads of R behind it, one dependent memory round trip per field.
__device__ __forceinline__ void step_scalars(const Rep& R, StepScalars& S) {
  S.adv = R.active && R.step < R.stop_step;
  S.step = R.step + 1;
  S.ens = (R.mode == kModePushoff) ? FMD_LANGEVIN : R.ensemble;
  const double dt = (R.mode == kModePushoff) ? R.push_dt : R.dt;
  S.dt = (float)dt;
  S.hdt = (float)(0.5 * dt);
  S.stream = (R.mode == kModePushoff) ? kStreamPushoff : kStreamLangevin;
  S.vscale = (float)R.pending_scale;
  S.ev = 1.0f;
  S.fpos = (float)dt;
  S.dh = 0.0f;
  S.h_new = R.h;
  S.h_old = R.h;
  S.inv_Lold = (float)(1.0 / R.Lpos);
  S.dW = 0.0f;
  S.L_new = R.L;
  S.nh = R.nh;
  if (S.ens == FMD_LANGEVIN) {
    const double kT = (R.mode == kModePushoff) ? R.T0 : ramp(R, S.step, R.T0, R.T1);
    const double c1 = (R.mode == kModePushoff) ? exp(-dt / R.Tdamp) : R.c1;
    S.c1 = (float)c1;
    S.c2kT = (float)(sqrt(1.0 - c1 * c1) * sqrt(kT));
  } else if (S.ens == FMD_NVT_NH) {
    const double kT = ramp(R, S.step, R.T0, R.T1);
    const double sc = nhc_half_step(S.nh.xi, S.nh.vxi, R.chain_M, R.Q1, R.Qr, kT, R.natoms, S.nh.carry, 0.5 * dt,
                                    S.nh.carry_dd ? S.nh.dd : nullptr);
    S.nh.scale = sc;
    S.vscale = (float)(R.pending_scale * sc);
  } else {
    const double kT = ramp(R, S.step, R.T0, R.T1), Pt = ramp(R, S.step, R.P0, R.P1);
    npt_chain_baro(S.nh, true, 0.0, 0.0, R.chain_M, R.Q1, R.Qr, R.W, 0.5 * dt, dt, R.V0, R.natoms, kT, Pt, DExp(),
                   DCbrt(), DSinh());
    S.vscale = (float)(R.pending_scale * (S.nh.scale * S.nh.bscale));
    S.ev = (float)S.nh.exp_vW;
    S.fpos = (float)S.nh.fpos;
    S.L_new = S.nh.L;
    const double hn = (double)(float)(S.nh.L / R.G);
    S.h_new = (float)hn;
    S.dh = (float)((double)R.h * S.nh.exp_vW - hn);
    // The reference scales positions wrapped into the previous box
    // (nose_hoover.cu:729-749 after the wrap of the step before); the scale
    // factor is not the box ratio, so an atom stored outside [0, L_old) picks
    // up w * (L_new - L_old * ev) per period w it lies outside.
    S.dW = (float)(S.nh.L - R.Lpos * S.nh.exp_vW);
  }
}

// R.next from R, built in a local and stored once.
__device__ __forceinline__ void next_scalars(Rep& R) {
  StepScalars nx;
  step_scalars(R, nx);
  R.next = nx;
}

// Three standard normals from the same Philox words as rng_normal3 (seed,
// stream, step, atom id), transformed in FP32: Box-Muller with u1 = (a + 1)
// 2^-32 and the angle split into quadrant (top two bits of b) and a quarter
// turn fraction, evaluated with the hardware-approximate __logf / __sincosf
// (absolute errors near 2^-21 on these ranges; the accurate logf / sincospif
// made the pre-force kernel 5 % slower).  Agrees with the FP64 transform to
// within those errors; the radius is clamped at zero, since near u1 = 1 the
// approximate logarithm's absolute error can exceed -ln u1 itself.
__device__ __forceinline__ void normal_pair_f32(uint32_t a, uint32_t b, float& z0, float& z1) {
  const float u1 = ((float)a + 1.0f) * 0x1.0p-32f;
  const float f = (float)(b & 0x3FFFFFFFu) * 0x1.0p-30f;
  float s, c;
  const float r = sqrtf(fmaxf(-2.0f * __logf(u1), 0.0f));
  __sincosf(1.5707963267948966f * f, &s, &c);
  const uint32_t q = b >> 30;
  const float cs = q == 0 ? c : (q == 1 ? -s : (q == 2 ? -c : s));
  const float sn = q == 0 ? s : (q == 1 ? c : (q == 2 ? -s : -c));
  z0 = r * cs;
  z1 = r * sn;
}

__device__ __forceinline__ void normal3_f32(uint64_t seed, uint32_t stream, uint64_t step, uint32_t id, float& n0,
                                            float& n1, float& n2) {
  U32x4 c;
  c.x = id;
  c.y = (uint32_t)step;
  c.z = (uint32_t)(step >> 32);
  c.w = stream;
  const U32x4 w = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  float z3;
  normal_pair_f32(w.x, w.y, n0, n1);
  normal_pair_f32(w.z, w.w, n2, z3);
}

__device__ __forceinline__ void warp_max_u32(uint32_t& v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
}


__device__ __forceinline__ void count_launch(const Dev& d, int kind) {
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(d.kcount + kind, 1ull);
}

// 16-byte asynchronous global -> shared copy (cp.async, L1-cached) and the
// wait for all of this thread's copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// The same copy with L1 bypassed (streamed data), the commit of this
// thread's copies issued so far as one group, and the wait until at most N
// of its groups are still in flight.
__device__ __forceinline__ void cp_async16_stream(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------- pre-force
// One atom's pre-force update on its loaded state (p, v, f, q); returns the
// squared displacement bits since the last rebuild and a non-finite flag.
__device__ __forceinline__ void pre_atom(const Dev& d, const Rep& R, const StepScalars& S, int s, bool deferred,
                                         float4 p, float4 v, const float4 f, float4 q, uint32_t& d2bits, int& bad) {
  const float hm = S.hdt * v.w;
  if (deferred) {
    // the previous step's post-force half kick (same step size, same
    // operation as the post-force kernel would have done)
    v.x = fmaf(hm, f.x, v.x);
    v.y = fmaf(hm, f.y, v.y);
    v.z = fmaf(hm, f.z, v.z);
  }
  v.x *= S.vscale;
  v.y *= S.vscale;
  v.z *= S.vscale;
  if (S.ens == FMD_LANGEVIN) {
    float n0, n1, n2;
    normal3_f32(R.seed, S.stream, (uint64_t)S.step, (uint32_t)__float_as_int(q.w), n0, n1, n2);
    const float ns = S.c2kT * sqrtf(v.w);
    v.x = fmaf(hm, f.x, v.x);
    v.y = fmaf(hm, f.y, v.y);
    v.z = fmaf(hm, f.z, v.z);
    p.x = fmaf(S.hdt, v.x, p.x);
    p.y = fmaf(S.hdt, v.y, p.y);
    p.z = fmaf(S.hdt, v.z, p.z);
    v.x = fmaf(S.c1, v.x, ns * n0);
    v.y = fmaf(S.c1, v.y, ns * n1);
    v.z = fmaf(S.c1, v.z, ns * n2);
    p.x = fmaf(S.hdt, v.x, p.x);
    p.y = fmaf(S.hdt, v.y, p.y);
    p.z = fmaf(S.hdt, v.z, p.z);
  } else if (S.ens == FMD_NVT_NH) {
    v.x = fmaf(hm, f.x, v.x);
    v.y = fmaf(hm, f.y, v.y);
    v.z = fmaf(hm, f.z, v.z);
    p.x = fmaf(S.dt, v.x, p.x);
    p.y = fmaf(S.dt, v.y, p.y);
    p.z = fmaf(S.dt, v.z, p.z);
  } else {
    v.x = fmaf(hm, f.x, v.x);
    v.y = fmaf(hm, f.y, v.y);
    v.z = fmaf(hm, f.z, v.z);
    const uint32_t u = w_bits(p.w);
    const float cx = (float)w_cx(u), cy = (float)w_cy(u), cz = (float)w_cz(u);
    const float wx = floorf(fmaf(cx, S.h_old, p.x) * S.inv_Lold);
    const float wy = floorf(fmaf(cy, S.h_old, p.y) * S.inv_Lold);
    const float wz = floorf(fmaf(cz, S.h_old, p.z) * S.inv_Lold);
    p.x = fmaf(p.x, S.ev, fmaf(cx, S.dh, fmaf(wx, S.dW, v.x * S.fpos)));
    p.y = fmaf(p.y, S.ev, fmaf(cy, S.dh, fmaf(wy, S.dW, v.y * S.fpos)));
    p.z = fmaf(p.z, S.ev, fmaf(cz, S.dh, fmaf(wz, S.dW, v.z * S.fpos)));
    q.x = fmaf(q.x, S.ev, cx * S.dh);
    q.y = fmaf(q.y, S.ev, cy * S.dh);
    q.z = fmaf(q.z, S.ev, cz * S.dh);
    d.ref[s] = q;
  }
  const float ux = p.x - q.x, uy = p.y - q.y, uz = p.z - q.z;
  const float dd = ux * ux + uy * uy + uz * uz;
  bad |= !isfinite(dd) || !isfinite(v.x + v.y + v.z);
  d2bits = max(d2bits, __float_as_uint(dd));
  d.pos[s] = p;
  d.vel[s] = v;
}

// Pre-force update of one chunk per block; each of the kChunk / APT threads
// updates APT atoms (all loads issued before any arithmetic).
template <int APT>
__global__ void __launch_bounds__(kChunk / APT, APT == 1 ? 12 : 16) k_pre(Dev d, StepConds cond) {
  constexpr int T = kChunk / APT;
  count_launch(d, kKPre);
  // the previous step's rebuild has finished: empty the work list before
  // this step's commits append to it
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d.rb[kRbCount] = 0;
    d.rb[kRbRebuilds] = 0;
    d.rb[kRbMode] = kRbNone;
  }
  // The atoms' data depends neither on the chunk's record nor on the replica
  // record or the step scalars: issue their loads first.  Chunk b holds slots
  // [b kChunk, (b + 1) kChunk), all allocated; the slots past the replica's
  // atoms (or of a free chunk) are loaded and left unused.
  const int base = blockIdx.x * kChunk;
  float4 p[APT], v[APT], f[APT], q[APT];
#pragma unroll
  for (int k = 0; k < APT; ++k) {
    const int t = threadIdx.x + k * T;
    p[k] = d.pos[base + t];
    v[k] = d.vel[base + t];
    f[k] = d.force[base + t];
    q[k] = d.ref[base + t];
  }
  const int4 ci = d.chunk_rep[blockIdx.x];
  if (ci.x < 0) return;
  Rep& R = d.reps[ci.x];
  __shared__ StepScalars S;
  __shared__ uint32_t wmax[T / 32];
  if (!(R.active && R.step < R.stop_step)) return;
  const bool deferred = R.defer != 0;
  // Every host upload is followed by k_prepare and every commit leaves
  // R.next valid, so a stale copy here is a fault, raised rather than
  // computed: an out-of-line call to compute it cost this kernel 18
  // registers, a stack frame and 4 blocks per SM.
  if (!R.next_valid) {
    if (threadIdx.x == 0) atomicOr(&R.status, kStatusStaleScalars);
    return;
  }
  {
    constexpr int nw = (int)(sizeof(StepScalars) / sizeof(uint32_t));
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&R.next);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&S);
    for (int k = threadIdx.x; k < nw; k += T) dst[k] = src[k];
  }
  __syncthreads();
  uint32_t d2bits = 0;
  int bad = 0;
#pragma unroll
  for (int k = 0; k < APT; ++k) {
    const int t = threadIdx.x + k * T;
    if (t < ci.z) pre_atom(d, R, S, base + t, deferred, p[k], v[k], f[k], q[k], d2bits, bad);
  }
  warp_max_u32(d2bits);
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = d2bits;
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    uint32_t m = 0;
    for (int w = 0; w < T / 32; ++w) m = max(m, wmax[w]);
    atomicMax(&R.maxdisp_bits, m);
    if (bad) atomicOr(&R.status, kStatusNonFinite);
  }
}

// Atoms per thread of the launched pre-force kernel: one (128 threads, 40
// registers, 12 blocks and 48 warps per SM) measured 0.9 % faster per step
// than two (64 threads, 62 registers, 16 blocks and 32 warps per SM).
constexpr int kPreAPT = 1;
constexpr int kPostCommitThreads = 512;  // per replica: the partials' reduction, then one thread commits

// Per-replica commit of the pre-force update (one thread per replica, after
// every pre-force block finished): step counter, chain / barostat state, box,
// the rebuild decision and the graph's conditional switches.
__device__ void commit_replica(const Dev& d, Rep& R, int r, const StepConds& cond);

__global__ void __launch_bounds__(32) k_commit(Dev d, StepConds cond) {
  count_launch(d, kKCommit);
  const int r = blockIdx.x;
  if (threadIdx.x != 0) return;
  if (r < d.rb_cap) {
    Rep& R = d.reps[r];
    if (R.active && R.step < R.stop_step) commit_replica(d, R, r, cond);  // advanced this step
  }
  // The last block chooses how this step rebuilds: the work-list kernels for
  // a few replicas, full grids (one block per chunk / home cell of every
  // replica) when many rebuild at once.
  __threadfence();
  if (atomicAdd(d.rb + kRbCommits, 1) != (int)gridDim.x - 1) return;
  __threadfence();
  d.rb[kRbCommits] = 0;
  const int n = d.rb[kRbCount], nr = d.rb[kRbRebuilds];
  const int mode = n == 0 ? kRbNone
                 : (nr == 0 ? kRbPrune : (nr >= kRbFullMin && 4 * nr >= (int)gridDim.x ? kRbFull : kRbList));
  d.rb[kRbMode] = mode;
  if (cond.use && mode == kRbList) cudaGraphSetConditional(cond.rebuild, 1u);
  if (cond.use && mode == kRbFull) cudaGraphSetConditional(cond.rebuild_full, 1u);
  if (cond.use && mode == kRbPrune) cudaGraphSetConditional(cond.prune, 1u);
}

__device__ void commit_replica(const Dev& d, Rep& R, int r, const StepConds& cond) {
  StepScalars S;
  if (R.next_valid) S = R.next;
  else step_scalars(R, S);
  R.next_valid = 0;
  R.step = S.step;
  R.nh = S.nh;
  R.pending_scale = 1.0;
  if (S.ens == FMD_NPT_NH) {
    R.L = S.L_new;
    R.h = S.h_new;
  }
  R.Lpos = R.L;
  R.adv = 1;
  R.since += 1;
  // An unlisted pair was farther than rc + skin when the list was built; an
  // NPT contraction by s since brings it to s (rc + skin) less the two atoms'
  // displacements in the co-scaled frame, so the list stays complete while
  // each displacement is below (s (rc + skin) - rc) / 2 (skin / 2 at
  // constant box, the trigger of skin_trigger.cuh:6-33).  Pairs inside the
  // box scale with the positions' factors, pairs across a face with the box:
  // s is the smaller of the two.
  if (S.ens == FMD_NPT_NH) {
    R.list_scale *= (double)S.ev;
    R.filter_scale *= (double)S.ev;
  }
  const float maxd2 = __uint_as_float(R.maxdisp_bits);
  const double s = fmin(R.L / R.L_list, R.list_scale);
  const float hs = (float)(s < 1.0 ? 0.5 * (s * (R.rc + R.skin) - R.rc) : 0.5 * R.skin);
  const bool trig = hs <= 0.f || maxd2 > hs * hs;
  // With a pruned list (pairs within rc + prune_delta), maxd2 is the
  // displacement since the last filter and disp_acc adds those of the earlier
  // filters: the full list's bound is their sum; the pruned list holds while
  // the displacement since its filter stays below (sp (rc + prune_delta) -
  // rc) / 2, sp the contraction since the filter (prune_delta / 2 at
  // constant box).  A rebuild filters its new list too.
  bool rtrig = trig;
  const float dmax = sqrtf(maxd2);
  if (R.disp_acc > 0.f) rtrig = hs <= 0.f || dmax + R.disp_acc > hs;
  const double sp = fmin(R.L / R.L_filter, R.filter_scale);
  const float hp = (float)(sp < 1.0 ? 0.5 * (sp * (R.rc + (double)R.prune_delta) - R.rc) : 0.5 * R.prune_delta);
  const bool ptrig = R.prune_delta > 0.f && (hp <= 0.f || dmax > hp);
  if (rtrig || R.since >= R.max_between) {
    R.since = 0;
    R.L_list = R.L;
    R.list_scale = 1.0;
    R.L_filter = R.L;
    R.filter_scale = 1.0;
    R.maxdisp_bits = 0u;
    R.disp_acc = 0.f;
    R.rebuilds += 1;
    R.rebuild_now = 1;
    atomicAdd(d.rb + kRbRebuilds, 1);
    d.rb[kRbHead + atomicAdd(d.rb + kRbCount, 1)] = r;
  } else if (ptrig) {
    R.disp_acc += dmax;
    R.maxdisp_bits = 0u;
    R.L_filter = R.L;
    R.filter_scale = 1.0;
    R.rebuild_now = 2;
    d.rb[kRbHead + atomicAdd(d.rb + kRbCount, 1)] = r;
  } else {
    R.rebuild_now = 0;
  }
  // Langevin steps inside a graph leave their post-force kick to the next
  // pre-force (the post-force kernel then has nothing else to do); the post
  // runs on energy steps, for the Nose-Hoover chains and on a replica's last
  // step of the run, so every state the host can read is complete.
  const bool langevin = R.mode == kModePushoff || R.ensemble == FMD_LANGEVIN;
  const bool post = !cond.use || !langevin || need_ev(R) || R.step >= R.stop_step;
  R.defer = post ? 0 : 1;
  if (cond.use) {
    // any replica that needs a force variant / a post switches it on
    if (need_ev(R)) cudaGraphSetConditional(cond.force_ev, 1u);  // the plain flavour is an unconditional node
    if (post) cudaGraphSetConditional(cond.post, 1u);
  }
  if (!post) {
    // a skipped post-force computes no scalars for the next step: do it here
    // (a Langevin post changes none of their inputs)
    next_scalars(R);
    R.next_valid = 1;
  }
}

// Scalars of the next pre-force for every active replica whose copy is
// stale (after a host upload), so that no pre-force block computes them.
__global__ void __launch_bounds__(32) k_prepare(Dev d) {
  count_launch(d, kKCommit);
  const int r = blockIdx.x;
  if (threadIdx.x != 0 || r >= d.rb_cap) return;
  Rep& R = d.reps[r];
  if (!R.active || R.next_valid) return;
  next_scalars(R);
  R.next_valid = 1;
}

// ---------------------------------------------------------------- rebuild
// Minimum-image cell shift of j relative to i and the periodic wrap count,
// for cell coordinates ci, cj and offsets oi, oj (one axis).
__device__ __forceinline__ void pair_shift(int ci, int cj, float oi, float oj, int G, float inv_h, int& e, int& k) {
  const int dc = ci - cj;
  const float D = (float)dc + (oi - oj) * inv_h;
  k = (int)rintf(D / (float)G);
  e = k * G - dc;
}

// Cell shift term e*h + k*dL (exact periodic box L = G*h + dL).
__device__ __forceinline__ float shift_term(int e, int k, float h, float dL) { return (float)e * h + (float)k * dL; }

// Neighbor-list work items: rows of kNbrRow home cells along x (G >= 3),
// single home cells for smaller grids.
constexpr int kNbrThreads = 128;
constexpr int kNbrRow = kNbrThreads / 32;  // home cells per item, one warp each
constexpr int kNbrCap = 1536;              // staged candidates (24 KB)
constexpr int kNbrUnion = (kNbrRow + 2) * 9;

__host__ __device__ inline int nbr_items(int G) { return G >= 3 ? G * G * ((G + kNbrRow - 1) / kNbrRow) : G * G * G; }

// ---- rebuild work list.  The pre-force kernel appends each replica that
// rebuilds this step; k_rbplan turns the list into prefix offsets of chunk
// and cell-group work items; the rebuild kernels run fixed grids that stride
// over those items only, so a step where a few replicas rebuild costs work
// for those replicas, not early exits over the whole batch.  The next step's
// pre-force kernel empties the list.
__device__ __forceinline__ int rb_count(const Dev& d) { return d.rb[kRbCount]; }
__device__ __forceinline__ int rb_rep(const Dev& d, int i) { return d.rb[kRbHead + i]; }
__device__ __forceinline__ int* rb_off(const Dev& d, int which) {
  return d.rb + kRbHead + d.rb_cap + which * (d.rb_cap + 1);
}

// index i with off[i] <= item < off[i + 1]
__device__ __forceinline__ int rb_find(const int* off, int n, int item) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= item) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Small single-block kernels (plans, per-replica scans) run kPlanThreads
// threads: blocks that fit beside the force kernels when they share the GPU.
constexpr int kPlanThreads = 256;

// Block-wide exclusive scan of v over the list (kPlanThreads threads), into off[0..n].
template <typename F>
__device__ void rb_scan(const Dev& d, int n, int* off, F value) {
  __shared__ int sm[kPlanThreads];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += kPlanThreads) {
    const int i = base + threadIdx.x;
    const int v = i < n ? value(rb_rep(d, i)) : 0;
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kPlanThreads; o <<= 1) {
      const int t = threadIdx.x >= o ? sm[threadIdx.x - o] : 0;
      __syncthreads();
      sm[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n) off[i] = carry + sm[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == kPlanThreads - 1) carry += sm[kPlanThreads - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) off[n] = carry;
}

constexpr int kCellGroup = 8;  // cells per cell-sort work item (one warp each)

// Offsets of chunk items and cell-group items (P^3 Morton cells per replica).
__global__ void __launch_bounds__(kPlanThreads) k_rbplan(Dev d) {
  count_launch(d, kKPlan);
  const int n = rb_count(d);
  // rebuild items count the rebuilding replicas only; the forces and the
  // list filter run over the chunks of every listed replica
  rb_scan(d, n, rb_off(d, 0), [&](int r) { return d.reps[r].rebuild_now == 1 ? d.reps[r].nchunks : 0; });
  rb_scan(d, n, rb_off(d, 1), [&](int r) {
    const int P = d.reps[r].P;
    return d.reps[r].rebuild_now == 1 ? (P * P * P + kCellGroup - 1) / kCellGroup : 0;
  });
  rb_scan(d, n, rb_off(d, 3), [&](int r) { return d.reps[r].nchunks; });
}

// Offsets of home-cell items (G^3 per replica, G as set by k_scan).
__global__ void __launch_bounds__(kPlanThreads) k_rbplan_home(Dev d, int variant) {
  count_launch(d, kKPlan);
  const int n = rb_count(d);
  rb_scan(d, n, rb_off(d, 2), [&](int r) {
    const int G = d.reps[r].G;
    if (d.reps[r].rebuild_now != 1 || G < 3) return 0;  // small boxes: k_neighbors_small
    return variant == 1 ? nbr_items(G) : G * G * G;
  });
}

// A block visits its items in increasing order, so the list entry of an item
// only moves forward: one search for the first item, then a step when an
// item passes the next offset.
struct RbCursor {
  const int* off;
  int n, i, lo, hi;
  __device__ __forceinline__ RbCursor(const int* o, int nn, int first) : off(o), n(nn), i(0), lo(0), hi(0) {
    if (n > 0 && first < off[n]) {
      i = rb_find(off, n, first);
      lo = off[i];
      hi = off[i + 1];
    }
  }
  __device__ __forceinline__ void seek(int item) {
    while (item >= hi) {
      ++i;
      lo = hi;
      hi = off[i + 1];
    }
  }
};

// Calls body(R, r, chunk index within the replica) for this block's chunk items.
template <typename F>
__device__ __forceinline__ void for_rebuild_chunks(const Dev& d, F body) {
  const int n = rb_count(d);
  const int* off = rb_off(d, 0);
  const int total = n > 0 ? off[n] : 0;
  RbCursor cur(off, n, blockIdx.x);
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    cur.seek(item);
    const int r = rb_rep(d, cur.i);
    body(d.reps[r], r, item - cur.lo);
  }
}

__device__ __forceinline__ void bin_chunk(const Dev& d, const Rep& R, int ci) {
  const int local = ci * kChunk + threadIdx.x;
  if (local >= R.natoms) return;
  const int s = R.slot_base + local;
  const float4 p = d.pos[s];
  int4 im = d.img[s];
  const uint32_t u = w_bits(p.w);
  const int c[3] = {w_cx(u), w_cy(u), w_cz(u)};
  const float o[3] = {p.x, p.y, p.z};
  const double L = R.L, h = (double)R.h;
  // New grid for the current box (re-derived at every rebuild).
  int Gn = (int)floor(L / ((R.rc + R.skin) * 1.0001));
  Gn = Gn < 1 ? 1 : (Gn > R.G_alloc ? R.G_alloc : Gn);
  const double hn = (double)(float)(L / Gn);
  int cn[3];
  float on[3];
  int dimg[3];
  for (int a = 0; a < 3; ++a) {
    double x = (double)c[a] * h + (double)o[a];
    int w = 0;
    if (x < 0.0) {
      x += L;
      w = -1;
    } else if (x >= L) {
      x -= L;
      w = 1;
    }
    int ca = (int)floor(x / hn);
    ca = ca < 0 ? 0 : (ca >= Gn ? Gn - 1 : ca);
    cn[a] = ca;
    on[a] = (float)(x - (double)ca * hn);
    dimg[a] = w;
  }
  im.x += dimg[0];
  im.y += dimg[1];
  im.z += dimg[2];
  const uint32_t key = cell_key(cn[0], cn[1], cn[2]);
  d.tpos[s] = make_float4(on[0], on[1], on[2], pack_w(cn[0], cn[1], cn[2], w_type(u)));
  d.timg[s] = im;
  d.tvel[s] = d.vel[s];
  d.key[s] = key;
  atomicAdd(&d.cell_cnt[R.cell_base + key], 1);
}

__global__ void __launch_bounds__(kChunk) k_bin(Dev d) {
  count_launch(d, kKBin);
  for_rebuild_chunks(d, [&](const Rep& R, int, int ci) { bin_chunk(d, R, ci); });
}

// Exclusive scan of the replica's cell counts; one block per replica.
// Cell offsets of a rebuilding replica: an exclusive scan of its cell counts
// (P^3 Morton-keyed cells; 262,144 at P = 64) by one block in tiles of
// kScanTile cells.  A tile is loaded and stored coalesced (lane-consecutive
// cells) and transposed through shared memory, so that each thread scans
// kScanPer consecutive cells; the next tile's counts are loaded while this
// one is scanned.  The shared index i is padded to i + i / 32, which keeps
// both access patterns free of bank conflicts.  (One pass of 256 threads
// over 1,024-cell strips took 0.9 ms at P = 64.)
constexpr int kScanThreads = 1024, kScanPer = 8, kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ int scan_pad(int i) { return i + (i >> 5); }

__global__ void __launch_bounds__(kScanThreads) k_scan(Dev d) {
  count_launch(d, kKScan);
  if ((int)blockIdx.x >= rb_count(d)) return;
  Rep& R = d.reps[rb_rep(d, blockIdx.x)];
  if (R.rebuild_now != 1) return;  // re-filters its pruned list only
  const int ncell = R.P * R.P * R.P;
  int* const cnt = d.cell_cnt + R.cell_base;
  int* const start = d.cell_start + R.cell_base;
  int* const fill = d.cell_fill + R.cell_base;
  __shared__ int s_t[kScanTile + kScanTile / 32];
  __shared__ int s_w[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int vn[kScanPer];
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) {
    const int c = j * kScanThreads + threadIdx.x;
    vn[j] = c < ncell ? cnt[c] : 0;
  }
  int carry = 0;
  for (int t0 = 0; t0 < ncell; t0 += kScanTile) {
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) s_t[scan_pad(j * kScanThreads + threadIdx.x)] = vn[j];
    if (t0 + kScanTile < ncell) {
#pragma unroll
      for (int j = 0; j < kScanPer; ++j) {
        const int c = t0 + kScanTile + j * kScanThreads + threadIdx.x;
        vn[j] = c < ncell ? cnt[c] : 0;
      }
    }
    __syncthreads();  // the tile is staged
    int v[kScanPer], sum = 0;
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
      v[j] = s_t[scan_pad(threadIdx.x * kScanPer + j)];
      sum += v[j];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += x;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int w = s_w[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xFFFFFFFFu, w, o);
        if (lane >= o) w += x;
      }
      s_w[lane] = w;
    }
    __syncthreads();
    int run = carry + (warp > 0 ? s_w[warp - 1] : 0) + incl - sum;
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
      s_t[scan_pad(threadIdx.x * kScanPer + j)] = run;
      run += v[j];
    }
    carry += s_w[kScanThreads / 32 - 1];
    __syncthreads();  // the offsets are staged
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
      const int k = j * kScanThreads + threadIdx.x;
      const int c = t0 + k;
      if (c < ncell) {
        const int o = s_t[scan_pad(k)];
        start[c] = o;
        fill[c] = o;
        cnt[c] = 0;
      }
    }
    __syncthreads();  // s_t and s_w are rewritten by the next tile
  }
  if (threadIdx.x == 0) {
    int Gn = (int)floor(R.L / ((R.rc + R.skin) * 1.0001));
    Gn = Gn < 1 ? 1 : (Gn > R.G_alloc ? R.G_alloc : Gn);
    R.G = Gn;
    R.h = (float)(R.L / Gn);
  }
}

__global__ void __launch_bounds__(kChunk) k_scatter(Dev d) {
  count_launch(d, kKScatter);
  for_rebuild_chunks(d, [&](const Rep& R, int, int ci) {
    const int local = ci * kChunk + threadIdx.x;
    if (local >= R.natoms) return;
    const int s = R.slot_base + local;
    const int at = atomicAdd(&d.cell_fill[R.cell_base + d.key[s]], 1);
    d.bucket[R.slot_base + at] = local;
  });
}

// Per cell: order members by atom id (deterministic), write the permutation.
// grid (cell blocks, replicas); one warp per cell.  Cells of up to 32
// members rank in registers with shuffles; larger ones fall back to a loop
// over the bucket.
__device__ __forceinline__ void cellsort_cell(const Dev& d, const Rep& R, int c, int lane) {
  {
    const int st = d.cell_start[R.cell_base + c];
    const int n = d.cell_fill[R.cell_base + c] - st;
    if (n <= 0) return;
    if (n <= 32) {
      int old = 0, id = 0x7FFFFFFF;
      if (lane < n) {
        old = d.bucket[R.slot_base + st + lane];
        id = d.timg[R.slot_base + old].w;
      }
      int rank = 0;
      for (int b = 0; b < n; ++b) rank += (__shfl_sync(0xFFFFFFFFu, id, b) < id);
      if (lane < n) d.perm[R.slot_base + st + rank] = old;
    } else {
      for (int a = lane; a < n; a += 32) {
        const int old = d.bucket[R.slot_base + st + a];
        const int id = d.timg[R.slot_base + old].w;
        int rank = 0;
        for (int b = 0; b < n; ++b) rank += (d.timg[R.slot_base + d.bucket[R.slot_base + st + b]].w < id);
        d.perm[R.slot_base + st + rank] = old;
      }
    }
  }
}

__global__ void __launch_bounds__(32 * kCellGroup) k_cellsort(Dev d) {
  count_launch(d, kKCellsort);
  const int n = rb_count(d);
  const int* off = rb_off(d, 1);
  const int total = n > 0 ? off[n] : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  RbCursor cur(off, n, blockIdx.x);
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    cur.seek(item);
    const Rep& R = d.reps[rb_rep(d, cur.i)];
    const int c = (item - cur.lo) * kCellGroup + warp;
    if (c < R.P * R.P * R.P) cellsort_cell(d, R, c, lane);
  }
}

__device__ __forceinline__ void permute_chunk(const Dev& d, const Rep& R, int ci) {
  const int local = ci * kChunk + threadIdx.x;
  const int s = R.slot_base + local;
  if (local >= R.natoms) {
    d.ncnt[s] = 0;
    return;
  }
  const int old = R.slot_base + d.perm[s];
  const float4 p = d.tpos[old];
  const int4 im = d.timg[old];
  d.pos[s] = p;
  d.ref[s] = make_float4(p.x, p.y, p.z, __int_as_float(im.w));
  d.vel[s] = d.tvel[old];
  d.img[s] = im;
  d.slot_of[R.slot_base + im.w] = local;
}

__global__ void __launch_bounds__(kChunk) k_permute(Dev d) {
  count_launch(d, kKPermute);
  for_rebuild_chunks(d, [&](const Rep& R, int, int ci) { permute_chunk(d, R, ci); });
}

// Per-slot bonded tables for the new order: partner slots instead of atom
// ids, so the force kernel reaches a partner's position in one load.
__device__ __forceinline__ void topo_chunk(const Dev& d, const Rep& R, int ci) {
  const int local = ci * kChunk + threadIdx.x;
  const int s = R.slot_base + local;
  if (local >= R.natoms) {
    d.tcnt[s] = 0;
    return;
  }
  const int base = R.slot_base;
  const int id = d.img[s].w;
  const int b0 = d.boff[base + id], b1 = d.boff[base + id + 1];
  const int a0 = d.aoff[base + id], a1 = d.aoff[base + id + 1];
  for (int b = b0; b < b1; ++b) {
    const int2 be = d.bent[R.bond_base + b];
    const uint32_t ps = (uint32_t)d.slot_of[base + be.x];
    d.bnd[(size_t)s * kMaxBondsPerAtom + (b - b0)] =
        ps | ((uint32_t)(be.y & 0xF) << 26) | ((uint32_t)((be.y >> 8) & 1) << 30);
  }
  for (int a = a0; a < a1; ++a) {
    const int4 ae = d.aent[R.angle_base + a];
    const int role = ae.w >> 8, ty = ae.w & 0xF;
    const uint32_t si = (uint32_t)d.slot_of[base + ae.x], sj = (uint32_t)d.slot_of[base + ae.y],
                   sk = (uint32_t)d.slot_of[base + ae.z];
    const uint32_t o1 = role == 0 ? sj : si;
    const uint32_t o2 = role == 2 ? sj : sk;
    d.ang[(size_t)s * kMaxAnglesPerAtom + (a - a0)] =
        make_uint2(o1 | ((uint32_t)role << 26), o2 | ((uint32_t)ty << 26));
  }
  d.tcnt[s] = (b1 - b0) | ((a1 - a0) << 8);
}

__global__ void __launch_bounds__(kChunk) k_topo(Dev d) {
  count_launch(d, kKTopo);
  for_rebuild_chunks(d, [&](const Rep& R, int, int ci) { topo_chunk(d, R, ci); });
}

// Verlet list for boxes of fewer than three cells per axis (L < 3 (rc +
// skin)): one warp per home cell, the distinct neighbor cells de-duplicated,
// each pair's periodic shift derived from the two cells and offsets.
// Candidates are broadcast 32 at a time with shuffles.
__device__ int neighbors_small_box(const Dev& d, Rep& R, int lc, int lane, int first = 0, int stride = 32) {
  const int G = R.G;
  const float h = R.h, inv_h = 1.0f / h;
  const float dL = (float)(R.L - (double)G * (double)h);
  const float rcs = (float)(R.rc + R.skin);
  const float rcs2 = rcs * rcs;
  const int M = R.M;
  const int base = R.slot_base;
  int overflow = 0;
  {
    const int hx = lc % G, hy = (lc / G) % G, hz = lc / (G * G);
    const uint32_t hkey = cell_key(hx, hy, hz);
    const int hs = d.cell_start[R.cell_base + hkey];
    const int he = d.cell_fill[R.cell_base + hkey];
    for (int hb = hs + first; hb < he; hb += stride) {
      const int il = hb + lane;
      const bool act = il < he;
      float4 pi = make_float4(0, 0, 0, 0);
      int idi = -1;
      int b0 = 0, b1 = 0;
      if (act) {
        pi = d.pos[base + il];
        idi = d.img[base + il].w;
        b0 = d.boff[base + idi];
        b1 = d.boff[base + idi + 1];
      }
      int count = 0;
      uint32_t* out = d.nbr + R.nbr_base + ((size_t)(il >> 5) * M) * 32 + (il & 31);
      int visited[27];  // distinct neighbor cells
      int nvis = 0;
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const int nx = (hx + dx + G) % G, ny = (hy + dy + G) % G, nz = (hz + dz + G) % G;
            const int lin = (nz * G + ny) * G + nx;
            bool seen = false;
            for (int v = 0; v < nvis; ++v) seen |= (visited[v] == lin);
            if (seen) continue;
            visited[nvis++] = lin;
            const uint32_t nkey = cell_key(nx, ny, nz);
            const int ns = d.cell_start[R.cell_base + nkey];
            const int ne = d.cell_fill[R.cell_base + nkey];
            for (int jb = ns; jb < ne; jb += 32) {
              const int jl = jb + lane;
              float4 pj = make_float4(0, 0, 0, 0);
              if (jl < ne) pj = d.pos[base + jl];
              const int m = min(32, ne - jb);
              for (int t = 0; t < m; ++t) {
                const float jx = __shfl_sync(0xFFFFFFFFu, pj.x, t);
                const float jy = __shfl_sync(0xFFFFFFFFu, pj.y, t);
                const float jz = __shfl_sync(0xFFFFFFFFu, pj.z, t);
                const float jw = __shfl_sync(0xFFFFFFFFu, pj.w, t);
                const int j = jb + t;
                if (!act || j == il) continue;
                int ex, ey, ez, kx, ky, kz;
                const uint32_t ui = w_bits(pi.w), uj = w_bits(jw);
                pair_shift(w_cx(ui), w_cx(uj), pi.x, jx, G, inv_h, ex, kx);
                pair_shift(w_cy(ui), w_cy(uj), pi.y, jy, G, inv_h, ey, ky);
                pair_shift(w_cz(ui), w_cz(uj), pi.z, jz, G, inv_h, ez, kz);
                const float rx = (pi.x - jx) - shift_term(ex, kx, h, dL);
                const float ry = (pi.y - jy) - shift_term(ey, ky, h, dL);
                const float rz = (pi.z - jz) - shift_term(ez, kz, h, dL);
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (r2 < rcs2) {
                  const int ax = axis_shift_code(ex, kx), ay = axis_shift_code(ey, ky), az = axis_shift_code(ez, kz);
                  if (ax < 0 || ay < 0 || az < 0) {
                    overflow |= kStatusCellCapacity;
                    continue;
                  }
                  const int idj = d.img[base + j].w;
                  bool excl = false;
                  for (int b = b0; b < b1; ++b) excl |= (d.bent[R.bond_base + b].x == idj);
                  if (excl) continue;
                  if (count < M)
                    out[(size_t)count * 32] = (uint32_t)j | entry_code(ax, ay, az);
                  ++count;
                }
              }
            }
          }
      if (act) {
        d.ncnt[base + il] = min(count, M);
        if (count > M) overflow |= kStatusOverflow;
        for (int k = count; k < ((count + kListPad - 1) & ~(kListPad - 1)) && k < M; ++k)
          out[(size_t)k * 32] = (uint32_t)il | kPadBits;
      }
    }
  }
  return overflow;
}

// Verlet list, ballot form: one block per home cell (G >= 3).  The 27 neighbor cells'
// atoms are staged in shared memory in stencil order (dz, dy, dx; slot order
// inside a cell) with the cell's periodic shift already added, so a pair's
// separation is one subtraction.  Each warp takes one home atom at a time;
// its lanes test 32 candidates, a ballot compacts the hits and they are
// stored in candidate order, so the list (and the force sums that follow it)
// is deterministic.  Pairs within rc + skin, 1-2 bonded pairs excluded
// (verlet_list.cu:108-335 semantics), exclusions compared as slots from the
// per-slot bond table.


constexpr int kNbrWarps = kNbrThreads / 32;
constexpr int kNbrWin = 1024;     // staged candidates per window
constexpr int kNbrGroup = 64;     // home atoms per pass

__device__ void neighbors_cell_ballot(const Dev& d, Rep& R, int lc) {
  const int G = R.G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (G < 3) return;  // boxes under three cells per axis: k_neighbors_small
  const int M = R.M;
  const int base = R.slot_base;
  const int cell_base = R.cell_base;
  uint32_t* const list = d.nbr + R.nbr_base;
  const float h = R.h;
  const float dL = (float)(R.L - (double)G * (double)h);
  const float rcs = (float)(R.rc + R.skin);
  const float rcs2 = rcs * rcs;

  __shared__ float4 s_c[kNbrWin];
  __shared__ int s_ns[27], s_off[28], s_cnt[kNbrGroup];
  __shared__ float s_sx[27], s_sy[27], s_sz[27];
  __shared__ uint32_t s_code[27];
  constexpr int kExcl = 1 + kMaxBondsPerAtom;  // the atom itself and its bonded partners
  __shared__ float4 s_hp[kNbrGroup];            // home atoms' positions
  __shared__ int s_xk[kNbrGroup][kExcl];        // and their excluded candidates (index, or -1)
  __shared__ uint32_t s_xm[kNbrWarps][kNbrWin / 32];  // per warp: excluded candidates of the window
  for (int k = threadIdx.x; k < kNbrWarps * (kNbrWin / 32); k += blockDim.x) (&s_xm[0][0])[k] = 0u;
  const int hx = lc % G, hy = (lc / G) % G, hz = lc / (G * G);
  if (warp == 0) {
    // the 27 cells (one lane each) and their candidate offsets (warp scan)
    int cnt = 0;
    if (lane < 27) {
      const int t = lane;
      const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
      const int nx = (hx + dx + G) % G, ny = (hy + dy + G) % G, nz = (hz + dz + G) % G;
      const uint32_t nkey = cell_key(nx, ny, nz);
      const int ns = d.cell_start[cell_base + nkey];
      s_ns[t] = ns;
      cnt = d.cell_fill[cell_base + nkey] - ns;
      // a candidate's position relative to the home cell: offset + shift
      const int kx = (hx + dx < 0) ? -1 : (hx + dx >= G ? 1 : 0);
      const int ky = (hy + dy < 0) ? -1 : (hy + dy >= G ? 1 : 0);
      const int kz = (hz + dz < 0) ? -1 : (hz + dz >= G ? 1 : 0);
      s_sx[t] = shift_term(dx, kx, h, dL);
      s_sy[t] = shift_term(dy, ky, h, dL);
      s_sz[t] = shift_term(dz, kz, h, dL);
      s_code[t] = entry_code(axis_shift_code(dx, kx), axis_shift_code(dy, ky), axis_shift_code(dz, kz));
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane < 27) s_off[lane + 1] = incl;
    if (lane == 0) s_off[0] = 0;
  }
  __syncthreads();
  const int total = s_off[27];
  const int hs = s_ns[13];
  const int nh = s_off[14] - s_off[13];
  if (nh == 0) return;
  int overflow = 0;
  const uint32_t lt = (1u << lane) - 1u;
  for (int hg = 0; hg < nh; hg += kNbrGroup) {
    const int gn = min(kNbrGroup, nh - hg);
    __syncthreads();  // the previous group's home data and window are no longer read
    // home atoms, one thread each (their loads in flight together): the
    // position, and the candidate indices of the atom itself and of its
    // bonded partners, whose cells (within one cell of the home cell: a bond
    // is shorter than a cell edge) the partners' cell fields give
    for (int a = threadIdx.x; a < gn; a += blockDim.x) {
      const int s = base + hs + hg + a;
      s_hp[a] = d.pos[s];
      s_xk[a][0] = s_off[13] + hg + a;
      const int nb = d.tcnt[s] & 0xFF;
#pragma unroll
      for (int b = 0; b < kMaxBondsPerAtom; ++b) {
        int k = -1;
        if (b < nb) {
          const int v = (int)(d.bnd[(size_t)s * kMaxBondsPerAtom + b] & kSlotMask26);
          const uint32_t u = w_bits(d.pos[base + v].w);
          int ex = w_cx(u) - hx, ey = w_cy(u) - hy, ez = w_cz(u) - hz;
          ex += ex > 1 ? -G : (ex < -1 ? G : 0);
          ey += ey > 1 ? -G : (ey < -1 ? G : 0);
          ez += ez > 1 ? -G : (ez < -1 ? G : 0);
          if (ex >= -1 && ex <= 1 && ey >= -1 && ey <= 1 && ez >= -1 && ez <= 1) {
            const int t = (ez + 1) * 9 + (ey + 1) * 3 + (ex + 1);
            if ((unsigned)(v - s_ns[t]) < (unsigned)(s_off[t + 1] - s_off[t])) k = s_off[t] + (v - s_ns[t]);
          }
        }
        s_xk[a][1 + b] = k;
      }
    }
    for (int w0 = 0; w0 < total; w0 += kNbrWin) {
      const int wn = min(kNbrWin, total - w0);
      if (hg == 0 || total > kNbrWin) {
        if (w0 > 0) __syncthreads();  // the previous window is no longer read
        // candidates of the window, each warp taking cells warp, warp + 4, ...:
        // asynchronous copies first (all in flight together), then each
        // thread adds the cell shifts to the candidates it copied
        for (int t = warp; t < 27; t += kNbrWarps) {
          const int o0 = s_off[t], o1 = s_off[t + 1];
          const int lo = max(o0, w0), hi = min(o1, w0 + wn);
          const float4* src = d.pos + base + s_ns[t] - o0;
          for (int k = lo + lane; k < hi; k += 32) cp_async16(&s_c[k - w0], src + k);
        }
        cp_async_wait_all();
        for (int t = warp; t < 27; t += kNbrWarps) {
          const int o0 = s_off[t], o1 = s_off[t + 1];
          const int lo = max(o0, w0), hi = min(o1, w0 + wn);
          const float sx = s_sx[t], sy = s_sy[t], sz = s_sz[t];
          const int ns = s_ns[t];
          const uint32_t code = s_code[t];
          for (int k = lo + lane; k < hi; k += 32) {
            const float4 p = s_c[k - w0];
            s_c[k - w0] = make_float4(p.x + sx, p.y + sy, p.z + sz, __uint_as_float((uint32_t)(ns + (k - o0)) | code));
          }
        }
      }
      // the window padded to whole pairs of 32 with candidates far away
      const int wnp = (wn + 63) & ~63;
      for (int k = wn + threadIdx.x; k < wnp; k += blockDim.x) s_c[k] = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
      __syncthreads();  // window (and home data) staged
      for (int a = warp; a < gn; a += kNbrWarps) {
        const int i = hs + hg + a;
        const float4 pi = s_hp[a];
        // this atom's excluded candidates in the window, as bits
        int xk = -1;
        if (lane < kExcl) {
          const int k = s_xk[a][lane] - w0;
          if (k >= 0 && k < wn) {
            xk = k;
            atomicOr(&s_xm[warp][k >> 5], 1u << (k & 31));
          }
        }
        __syncwarp();
        int count = w0 == 0 ? 0 : s_cnt[a];
        uint32_t* out = list + ((size_t)(i >> 5) * M) * 32 + (i & 31);
#pragma unroll 2
        for (int c0 = 0; c0 < wnp; c0 += 32) {
          const float4 c = s_c[c0 + lane];
          const float rx = pi.x - c.x, ry = pi.y - c.y, rz = pi.z - c.z;
          const float r2 = rx * rx + ry * ry + rz * rz;
          const uint32_t m = __ballot_sync(0xFFFFFFFFu, r2 < rcs2) & ~s_xm[warp][c0 >> 5];
          const int at = count + __popc(m & lt);
          if (((m >> lane) & 1u) && at < M) __stcg(out + (size_t)at * 32, __float_as_uint(c.w));
          count += __popc(m);
        }
        __syncwarp();
        if (xk >= 0) s_xm[warp][xk >> 5] = 0u;
        __syncwarp();
        if (w0 + kNbrWin >= total) {
          if (count <= M) {
            const int padded = (count + kListPad - 1) & ~(kListPad - 1);
            if (lane < padded - count)
              __stcg(out + (size_t)(count + lane) * 32, (uint32_t)i | kPadBits);
          }
          if (lane == 0) {
            d.ncnt[base + i] = min(count, M);
            if (count > M) overflow |= kStatusOverflow;
          }
        } else if (lane == 0) {
          s_cnt[a] = count;
        }
      }
    }
  }
  if (overflow) atomicOr(&R.status, overflow);
}

// Verlet list (G >= 3): one block per row of up to kNbrRow home cells along
// x.  The union of their neighbor cells (a (row + 2) x 3 x 3 block of cells)
// is staged once in shared memory, each candidate with its cell's periodic
// shift relative to the row origin already added; cells beyond the staging
// capacity are read from global memory instead.  Each warp owns one home
// cell, its lanes are that cell's atoms (32 at a time), and it walks its own
// 27 cells in stencil order (dz, dy, dx; slot order inside a cell) with every
// lane reading the same candidate (shared-memory broadcast); hits are
// appended per lane, so each list is in candidate order and deterministic.
// Pairs within rc + skin, 1-2 bonded pairs excluded (verlet_list.cu:108-335
// semantics), exclusions compared as slots from the per-slot bond table.

__device__ void neighbors_row(const Dev& d, Rep& R, int item) {
  const int G = R.G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (G < 3) return;  // boxes under three cells per axis: k_neighbors_small
  const int nrow = (G + kNbrRow - 1) / kNbrRow;
  const int bx = item % nrow, hy = (item / nrow) % G, hz = item / (nrow * G);
  const int hx0 = bx * kNbrRow;
  const int nhome = min(kNbrRow, G - hx0);
  const int ux = nhome + 2;  // union columns: x = hx0 - 1 ... hx0 + nhome
  const int nu = ux * 9;
  const int M = R.M;
  const int base = R.slot_base;
  const int cell_base = R.cell_base;
  uint32_t* const list = d.nbr + R.nbr_base;
  const float h = R.h;
  const float dL = (float)(R.L - (double)G * (double)h);
  const float rcs = (float)(R.rc + R.skin);
  const float rcs2 = rcs * rcs;

  __shared__ float4 s_c[kNbrCap];
  __shared__ int s_ns[kNbrUnion], s_off[kNbrUnion + 1];
  __shared__ float s_sx[kNbrUnion], s_sy[kNbrUnion], s_sz[kNbrUnion];
  __shared__ int s_ax[kNbrUnion];   // wrap count kx of the union column
  __shared__ uint32_t s_ayz[kNbrUnion];  // the y and z axis codes' fields of the entry
  if (threadIdx.x < nu) {
    const int u = threadIdx.x;
    const int row = u / ux, col = u % ux;
    const int dz = row / 3 - 1, dy = row % 3 - 1;
    const int xu = hx0 - 1 + col;
    const int kx = xu < 0 ? -1 : (xu >= G ? 1 : 0);
    const int ky = hy + dy < 0 ? -1 : (hy + dy >= G ? 1 : 0);
    const int kz = hz + dz < 0 ? -1 : (hz + dz >= G ? 1 : 0);
    const int nx = xu - kx * G, ny = hy + dy - ky * G, nz = hz + dz - kz * G;
    const uint32_t key = cell_key(nx, ny, nz);
    const int ns = d.cell_start[cell_base + key];
    s_ns[u] = ns;
    s_off[u + 1] = d.cell_fill[cell_base + key] - ns;
    // relative to the row origin: x shift (xu - hx0) h + kx dL
    s_sx[u] = shift_term(xu - hx0, kx, h, dL);
    s_sy[u] = shift_term(dy, ky, h, dL);
    s_sz[u] = shift_term(dz, kz, h, dL);
    s_ax[u] = kx;
    s_ayz[u] = entry_code(0, axis_shift_code(dy, ky), axis_shift_code(dz, kz));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s_off[0] = 0;
    for (int u = 0; u < nu; ++u) s_off[u + 1] += s_off[u];
  }
  __syncthreads();
  const int staged = min(s_off[nu], kNbrCap);
  for (int u = warp; u < nu; u += kNbrRow) {
    const int o0 = s_off[u], o1 = min(s_off[u + 1], kNbrCap);
    const float sx = s_sx[u], sy = s_sy[u], sz = s_sz[u];
    const int ns = s_ns[u];
    for (int k = o0 + lane; k < o1; k += 32) {
      const int j = ns + (k - o0);
      const float4 p = d.pos[base + j];
      s_c[k] = make_float4(p.x + sx, p.y + sy, p.z + sz, __int_as_float(j));
    }
  }
  __syncthreads();
  int overflow = 0;
  if (warp < nhome) {
    const int a = warp;  // this warp's home cell: x = hx0 + a
    const int uh = 4 * ux + a + 1;
    const int hs = s_ns[uh];
    const int nh = s_off[uh + 1] - s_off[uh];
    const float ah = (float)a * h;
    for (int hb = 0; hb < nh; hb += 32) {
      const bool act = hb + lane < nh;
      const int i = hs + hb + lane;
      float4 pi = make_float4(0, 0, 0, 0);
      uint32_t ex0 = 0xFFFFFFFFu, ex1 = ex0, ex2 = ex0, ex3 = ex0;
      if (act) {
        pi = d.pos[base + i];
        pi.x += ah;
        const int nb = d.tcnt[base + i] & 0xFF;
        const uint32_t* bl = d.bnd + (size_t)(base + i) * kMaxBondsPerAtom;
        if (nb > 0) ex0 = bl[0] & kSlotMask26;
        if (nb > 1) ex1 = bl[1] & kSlotMask26;
        if (nb > 2) ex2 = bl[2] & kSlotMask26;
        if (nb > 3) ex3 = bl[3] & kSlotMask26;
      }
      uint32_t* out = list + ((size_t)(i >> 5) * M) * 32 + (i & 31);
      int count = 0;
      for (int row = 0; row < 9; ++row) {
        for (int dx = -1; dx <= 1; ++dx) {
          const int u = row * ux + a + 1 + dx;
          const uint32_t code = entry_code(axis_shift_code(dx, s_ax[u]), 0, 0) | s_ayz[u];
          const int k0 = s_off[u], k1 = s_off[u + 1];
          const float sx = s_sx[u], sy = s_sy[u], sz = s_sz[u];
          const int ns = s_ns[u];
#pragma unroll 4
          for (int k = k0; k < k1; ++k) {
            float4 c;
            if (k < staged) {
              c = s_c[k];
            } else {
              const int j = ns + (k - k0);
              const float4 p = d.pos[base + j];
              c = make_float4(p.x + sx, p.y + sy, p.z + sz, __int_as_float(j));
            }
            const uint32_t j = (uint32_t)__float_as_int(c.w);
            const float rx = pi.x - c.x, ry = pi.y - c.y, rz = pi.z - c.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            const bool hit = act && r2 < rcs2 && j != (uint32_t)i && j != ex0 && j != ex1 && j != ex2 && j != ex3;
            if (hit && count < M) __stcg(out + (size_t)count * 32, j | code);
            count += hit ? 1 : 0;
          }
        }
      }
      if (act) {
        d.ncnt[base + i] = min(count, M);
        if (count > M) {
          overflow |= kStatusOverflow;
        } else {
          for (int k = count; k < ((count + kListPad - 1) & ~(kListPad - 1)); ++k)
            __stcg(out + (size_t)k * 32, (uint32_t)i | kPadBits);
        }
      }
    }
  }
  if (overflow) atomicOr(&R.status, overflow);
}

// Neighbor-list kernel variants: V = 0 ballot form (one home cell per item),
// V = 1 row form (kNbrRow home cells per item); MINB = blocks per SM the
// registers are fitted to.  The autotuner picks one.
template <int V, int MINB>
__global__ void __launch_bounds__(kNbrThreads, MINB) k_neighbors(Dev d) {
  count_launch(d, kKNeighbors);
  const int n = rb_count(d);
  const int* off = rb_off(d, 2);
  const int total = n > 0 ? off[n] : 0;
  RbCursor cur(off, n, blockIdx.x);
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    cur.seek(item);
    __syncthreads();  // the previous item's shared staging is no longer read
    if (V == 0)
      neighbors_cell_ballot(d, d.reps[rb_rep(d, cur.i)], item - cur.lo);
    else
      neighbors_row(d, d.reps[rb_rep(d, cur.i)], item - cur.lo);
  }
}

// Lists of the rebuilding replicas whose box holds fewer than three cells
// per axis (L < 3 (rc + skin), a few hundred beads): one block per (home
// cell, work-list replica) -- G <= 2, so at most 8 cells -- its warps taking
// the cell's home atoms 32 at a time in turn with the de-duplicated small-box
// form (each list is its lane's own: the split changes no entry).  The ballot
// and row kernels skip those replicas, which keeps the small form's
// dynamically indexed cell list (a stack frame) out of their registers: 72
// instead of 80 at 6 blocks per SM, and no spill at 8.  (One warp walking a
// replica's 8 cells in turn made a 500-bead replica's rebuild the long pole
// of the step: 256 uneven replicas fell from 3.0e9 to 1.8e9 atom-steps/s.)
constexpr int kSmallWarps = 4;

__global__ void __launch_bounds__(32 * kSmallWarps) k_neighbors_small(Dev d) {
  if ((int)blockIdx.y >= rb_count(d)) return;
  Rep& R = d.reps[rb_rep(d, blockIdx.y)];
  const int G = R.G;
  if (R.rebuild_now != 1 || G >= 3) return;
  const int lc = blockIdx.x;
  if (lc >= G * G * G) return;
  const int ov = neighbors_small_box(d, R, lc, threadIdx.x & 31, 32 * (threadIdx.x >> 5), 32 * kSmallWarps);
  if (ov) atomicOr(&R.status, ov);
}

// ---------------------------------------------------------------- forces

struct KahanF {
  float s, c;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// One axis of r_i - r_j for a bonded pair.  A bond is shorter than a cell
// edge and cells are fixed between rebuilds, so the two cells differ by at
// most one modulo the periodic wrap: for G >= 3 the shift follows from the
// cell indices alone (integer arithmetic); smaller grids take the general
// offset-based form.  Both give the same e, k and hence the same value.
__device__ __forceinline__ float bonded_axis(int ci, int cj, float oi, float oj, int G, float h, float inv_h,
                                             float dL) {
  int e, k;
  if (G >= 3) {
    const int dc = ci - cj;
    k = dc > 1 ? 1 : (dc < -1 ? -1 : 0);
    e = k * G - dc;
  } else {
    pair_shift(ci, cj, oi, oj, G, inv_h, e, k);
  }
  return (oi - oj) - shift_term(e, k, h, dL);
}

__device__ __forceinline__ float3 bonded_dr(float4 pi, float4 pj, int G, float h, float inv_h, float dL) {
  const uint32_t ui = w_bits(pi.w), uj = w_bits(pj.w);
  return make_float3(bonded_axis(w_cx(ui), w_cx(uj), pi.x, pj.x, G, h, inv_h, dL),
                     bonded_axis(w_cy(ui), w_cy(uj), pi.y, pj.y, G, h, inv_h, dL),
                     bonded_axis(w_cz(ui), w_cz(uj), pi.z, pj.z, G, h, inv_h, dL));
}

template <int BS>
__device__ __forceinline__ void block_partials(double* vals, int nv, double* out, int64_t stride) {
  __shared__ double sm[BS / 32][8];
  for (int c = 0; c < nv; ++c) vals[c] = warp_sum(vals[c]);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < nv; ++c) sm[threadIdx.x >> 5][c] = vals[c];
  __syncthreads();
  if (threadIdx.x < nv) {
    double t = 0.0;
    for (int w = 0; w < BS / 32; ++w) t += sm[w][threadIdx.x];
    out[threadIdx.x * stride] = t;
  }
}

// LJ contribution of one listed neighbor (lj.cu:32-61 semantics).  sh is
// the periodic shift vector named by the entry's code, so
// r_ij = (pos_i - pos_j) - sh.  EV: also accumulate half the pair energy and
// the virial half-pair.
struct PairAcc {
  float fx, fy, fz, pe, v0, v1, v2, v3, v4, v5;
};

// Every force path evaluates a pair with the same sequence of correctly
// rounded operations (explicit intrinsics, no contraction left to the
// compiler), so the packed two-pair form below, the scalar form, the energy
// flavour and the list filter give bit-identical forces for one variant.
__device__ __forceinline__ float pair_r2(float4 pi, float3 sh, float4 pj, float& dx, float& dy, float& dz) {
  dx = __fsub_rn(__fsub_rn(pi.x, pj.x), sh.x);
  dy = __fsub_rn(__fsub_rn(pi.y, pj.y), sh.y);
  dz = __fsub_rn(__fsub_rn(pi.z, pj.z), sh.z);
  return __fmaf_rn(dz, dz, __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
}

// F/r of a pair at r2 (lj.cu:32-61: 24 eps r^-2 (2 (s/r)^12 - (s/r)^6), clamped
// to +-1000 as lj.cu:48 does); pairs at or beyond the cutoff (padding entries
// included) give an exact zero.  The reference also skips r^2 <= 1e-10
// (coincident atoms); here such a pair's F/r clamps to +-1000 times a
// separation below 1e-5, and only its energy is left out.
// 1 / r^2 of a pair: the approximate reciprocal instruction alone (r^2 is
// never subnormal: a listed pair's r^2 lies between the overlap clamp and
// (rc + skin)^2, a padding entry's near 3 (h + dL)^2; r^2 = 0 gives +inf,
// which the force clamp turns into +-1000 as before).  The force launch at
// 64 x 30K is 2-4 % faster than with the fast-divide intrinsic, whose range
// scaling the pair loop never needs.
__device__ __forceinline__ float recip_r2(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float lj_fr(float r2, float rc2, float e24, float sig2, float& inv, float& sr6) {
  inv = recip_r2(r2);
  const float sr2 = __fmul_rn(sig2, inv);
  sr6 = __fmul_rn(__fmul_rn(sr2, sr2), sr2);
  const float t = __fmaf_rn(sr6, 2.0f, -1.0f);
  const float fr = __fmul_rn(__fmul_rn(__fmul_rn(e24, inv), sr6), t);
  return r2 < rc2 ? fminf(fmaxf(fr, -1000.0f), 1000.0f) : 0.0f;
}

template <bool EV>
__device__ __forceinline__ void lj_pair(PairAcc& a, float4 pi, float3 sh, float4 pj, float rc2, float e24,
                                        float sig2) {
  float dx, dy, dz, inv, sr6;
  const float r2 = pair_r2(pi, sh, pj, dx, dy, dz);
  const float fr = lj_fr(r2, rc2, e24, sig2, inv, sr6);
  a.fx = __fmaf_rn(fr, dx, a.fx);
  a.fy = __fmaf_rn(fr, dy, a.fy);
  a.fz = __fmaf_rn(fr, dz, a.fz);
  if (EV) {
    const float fxij = fr * dx, fyij = fr * dy, fzij = fr * dz;
    const bool in = r2 < rc2;
    const float e = in && r2 > 1e-10f ? e24 * (1.0f / 12.0f) * (sr6 * (sr6 - 1.0f)) : 0.0f;  // 1/2 * 4 eps (sr12 - sr6)
    a.pe += e;
    a.v0 = fmaf(fxij, dx, a.v0);
    a.v1 = fmaf(fxij, dy, a.v1);
    a.v2 = fmaf(fxij, dz, a.v2);
    a.v3 = fmaf(fyij, dy, a.v3);
    a.v4 = fmaf(fyij, dz, a.v4);
    a.v5 = fmaf(fzij, dz, a.v5);
  }
}

// Packed FP32x2 arithmetic (sm_100): two independent IEEE operations per
// instruction, each lane rounded exactly as the scalar operation.
__device__ __forceinline__ float2 sub_f32x2(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 ra, rb, rr;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rr, ra, rb;\n\tmov.b64 {%0, %1}, rr;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

// Forces of two list entries in packed FP32x2 form: the (x, y) components of
// a pair together, then the two pairs' scalar factors together.  Bitwise the
// same as two lj_pair<false> calls in entry order.
__device__ __forceinline__ void lj_pair2(PairAcc& a, float4 pi, float3 sha, float4 pja, float3 shb, float4 pjb,
                                         float rc2, float e24, float sig2) {
  const float2 pxy = make_float2(pi.x, pi.y);
  const float2 dxya = sub_f32x2(sub_f32x2(pxy, make_float2(pja.x, pja.y)), make_float2(sha.x, sha.y));
  const float2 dxyb = sub_f32x2(sub_f32x2(pxy, make_float2(pjb.x, pjb.y)), make_float2(shb.x, shb.y));
  const float dza = __fsub_rn(__fsub_rn(pi.z, pja.z), sha.z);
  const float dzb = __fsub_rn(__fsub_rn(pi.z, pjb.z), shb.z);
  const float2 ma = __fmul2_rn(dxya, dxya), mb = __fmul2_rn(dxyb, dxyb);
  const float2 r2 = make_float2(__fmaf_rn(dza, dza, __fadd_rn(ma.x, ma.y)), __fmaf_rn(dzb, dzb, __fadd_rn(mb.x, mb.y)));
  const float2 inv = make_float2(recip_r2(r2.x), recip_r2(r2.y));
  const float2 sr2 = __fmul2_rn(make_float2(sig2, sig2), inv);
  const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
  const float2 t = __ffma2_rn(sr6, make_float2(2.0f, 2.0f), make_float2(-1.0f, -1.0f));
  const float2 fr2 = __fmul2_rn(__fmul2_rn(__fmul2_rn(make_float2(e24, e24), inv), sr6), t);
  const float fa = r2.x < rc2 ? fminf(fmaxf(fr2.x, -1000.0f), 1000.0f) : 0.0f;
  const float fb = r2.y < rc2 ? fminf(fmaxf(fr2.y, -1000.0f), 1000.0f) : 0.0f;
  float2 g = __ffma2_rn(make_float2(fa, fa), dxya, make_float2(a.fx, a.fy));
  a.fz = __fmaf_rn(fa, dza, a.fz);
  g = __ffma2_rn(make_float2(fb, fb), dxyb, g);
  a.fz = __fmaf_rn(fb, dzb, a.fz);
  a.fx = g.x;
  a.fy = g.y;
}

// Periodic shift vector of a list entry.  SH = 0: the entry's 3D vector from
// the 125-entry table (index 25 ax + 5 ay + az; one 16-byte shared load,
// whose lanes conflict across banks).  SH = 1: each axis value from the
// 5-value table (three 4-byte shared loads that never conflict: the table
// spans 5 banks).  The same values either way.
template <int SH>
__device__ __forceinline__ float3 entry_shift(uint32_t w, const float4* s_shift, const float* s_axis) {
  const int ax = entry_ax(w), ay = entry_ay(w), az = entry_az(w);
  if (SH == 0) {
    const float4 v = s_shift[25 * ax + 5 * ay + az];
    return make_float3(v.x, v.y, v.z);
  }
  return make_float3(s_axis[ax], s_axis[ay], s_axis[az]);
}

// The LJ loop over one atom's list in batches of B entries: all list loads,
// then all position gathers, then the arithmetic.  PF: the next batch's list
// words are loaded before this batch's gathers (software pipelining, B more
// registers).  nn is the padded length (a multiple of B).  LPA lanes per
// atom: this lane walks the batches starting at entry k0 = (its lane group)
// * B, every LPA-th batch.
template <bool EV, int B, bool PF, int KB, bool ONE, int SH, bool P2, int LPA = 1>
__device__ __forceinline__ void lj_loop(const uint32_t* lst, int nn, const float4* pbase, float4 pi,
                                        const float4* s_shift, const float* s_axis, int ti, int nt,
                                        const float* s_eps24, const float* s_sig2, float rc2, KahanF& fx, KahanF& fy,
                                        KahanF& fz, PairAcc& acc, int k0 = 0) {
  constexpr int STEP = B * LPA;
  const float e24_0 = s_eps24[0], sig2_0 = s_sig2[0];
  uint32_t wn[B];
  if (PF) {
#pragma unroll
    for (int q = 0; q < B; ++q) wn[q] = nn > k0 ? __ldg(lst + (size_t)(k0 + q) * 32) : 0u;
  }
  // plain sums over KB batches (KB * B <= 8 pairs), then one compensated add
  PairAcc g = {0, 0, 0, acc.pe, acc.v0, acc.v1, acc.v2, acc.v3, acc.v4, acc.v5};
  int kb = 0;
  for (int k = k0; k < nn; k += STEP) {
    uint32_t w[B];
    if (PF) {
#pragma unroll
      for (int q = 0; q < B; ++q) w[q] = wn[q];
      if (k + STEP < nn) {
#pragma unroll
        for (int q = 0; q < B; ++q) wn[q] = __ldg(lst + (size_t)(k + STEP + q) * 32);
      }
    } else {
#pragma unroll
      for (int q = 0; q < B; ++q) w[q] = __ldg(lst + (size_t)(k + q) * 32);
    }
    float4 pj[B];
#pragma unroll
    for (int q = 0; q < B; ++q) pj[q] = __ldg(pbase + (w[q] & kIdxMask));
    if (P2 && ONE && !EV) {
#pragma unroll
      for (int q = 0; q < B; q += 2)
        lj_pair2(g, pi, entry_shift<SH>(w[q], s_shift, s_axis), pj[q], entry_shift<SH>(w[q + 1], s_shift, s_axis),
                 pj[q + 1], rc2, e24_0, sig2_0);
    } else {
#pragma unroll
      for (int q = 0; q < B; ++q) {
        float e24 = e24_0, sig2 = sig2_0;
        if (!ONE) {
          const int pidx = ti * nt + w_type(w_bits(pj[q].w));
          e24 = s_eps24[pidx];
          sig2 = s_sig2[pidx];
        }
        lj_pair<EV>(g, pi, entry_shift<SH>(w[q], s_shift, s_axis), pj[q], rc2, e24, sig2);
      }
    }
    if (++kb == KB || k + STEP >= nn) {
      fx.add(g.fx);
      fy.add(g.fy);
      fz.add(g.fz);
      g.fx = g.fy = g.fz = 0.0f;
      kb = 0;
    }
  }
  acc.pe = g.pe;
  acc.v0 = g.v0;
  acc.v1 = g.v1;
  acc.v2 = g.v2;
  acc.v3 = g.v3;
  acc.v4 = g.v4;
  acc.v5 = g.v5;
}

// The LJ loop with the list rows staged through a shared-memory ring of D
// batches per warp.  A warp's 32 atoms share one 32-slot tile of the
// transposed list, whose rows (128 bytes: entry k of the 32 atoms) are
// contiguous, so a batch of 4 rows (512 bytes) is fetched by one 16-byte
// asynchronous copy per lane (L1 bypassed), D - 1 batches ahead of its use
// (D - 2 while it is read), without registers held for it; each lane then
// reads its own words from shared memory.  The warp walks its longest list (nmax, warp-uniform): a
// lane's entries past its own length nn read as its padding entry and its
// compensated adds stop at nn, so the forces are bitwise those of lj_loop
// with B = 4 and the same KB, SH and P2.
template <bool EV, int KB, bool ONE, int SH, bool P2, int D>
__device__ __forceinline__ void lj_loop_ring(const uint32_t* tile_rows, uint32_t* ring, int lane, int nn, int nmax,
                                             uint32_t pad, const float4* pbase, float4 pi, const float4* s_shift,
                                             const float* s_axis, int ti, int nt, const float* s_eps24,
                                             const float* s_sig2, float rc2, KahanF& fx, KahanF& fy, KahanF& fz,
                                             PairAcc& acc) {
  constexpr int B = 4;
  constexpr int W = B * 32;  // words per batch
  const float e24_0 = s_eps24[0], sig2_0 = s_sig2[0];
  const int nb = nmax / B;
  // batches 0 .. D - 2 in flight before the loop; batch b + D - 1 is issued
  // once batch b has landed, into the slot batch b - 1 was read from
  const uint32_t* src = tile_rows + lane * 4;
  uint32_t* const dst = ring + lane * 4;
#pragma unroll
  for (int b = 0; b < D - 1; ++b) {
    if (b < nb) cp_async16_stream(dst + b * W, src);
    cp_async_commit();
    src += W;
  }
  PairAcc g = {0, 0, 0, acc.pe, acc.v0, acc.v1, acc.v2, acc.v3, acc.v4, acc.v5};
  int kb = 0;
  int rd = 0, wr = D - 1;  // ring slots of batch b and of batch b + D - 1
  for (int b = 0; b < nb; ++b) {
    cp_async_wait_group<D - 2>();  // this lane's part of batch b has landed
    __syncwarp();  // every lane's part has, and every lane is done reading slot wr (batch b - 1)
    if (b + D - 1 < nb) cp_async16_stream(dst + wr * W, src);
    cp_async_commit();
    src += W;
    const uint32_t* slot = ring + rd * W;
    rd = rd + 1 == D ? 0 : rd + 1;
    wr = wr + 1 == D ? 0 : wr + 1;
    const int k = b * B;
    uint32_t w[B];
#pragma unroll
    for (int q = 0; q < B; ++q) w[q] = k + q < nn ? slot[q * 32 + lane] : pad;
    float4 pj[B];
#pragma unroll
    for (int q = 0; q < B; ++q) pj[q] = __ldg(pbase + (w[q] & kIdxMask));
    if (P2 && ONE && !EV) {
#pragma unroll
      for (int q = 0; q < B; q += 2)
        lj_pair2(g, pi, entry_shift<SH>(w[q], s_shift, s_axis), pj[q], entry_shift<SH>(w[q + 1], s_shift, s_axis),
                 pj[q + 1], rc2, e24_0, sig2_0);
    } else {
#pragma unroll
      for (int q = 0; q < B; ++q) {
        float e24 = e24_0, sig2 = sig2_0;
        if (!ONE) {
          const int pidx = ti * nt + w_type(w_bits(pj[q].w));
          e24 = s_eps24[pidx];
          sig2 = s_sig2[pidx];
        }
        lj_pair<EV>(g, pi, entry_shift<SH>(w[q], s_shift, s_axis), pj[q], rc2, e24, sig2);
      }
    }
    if (k < nn && (++kb == KB || k + B >= nn)) {
      fx.add(g.fx);
      fy.add(g.fy);
      fz.add(g.fz);
      g.fx = g.fy = g.fz = 0.0f;
      kb = 0;
    }
  }
  cp_async_wait_group<0>();
  acc.pe = g.pe;
  acc.v0 = g.v0;
  acc.v1 = g.v1;
  acc.v2 = g.v2;
  acc.v3 = g.v3;
  acc.v4 = g.v4;
  acc.v5 = g.v5;
}

// The LJ loop of a replica whose pruned list is due (rebuilt or filtered this
// step), fused with the filter: it walks the rc + skin list, evaluates the
// entries within rc + prune_delta (the others lie beyond rc and contribute
// nothing) and writes them, in list order and padded, as the new pruned list.
// The compensated adds follow the pruned list's batches (one per B * KB kept
// entries, then those of its padding), so the forces are bit-identical to a
// walk of the list it writes: a later re-evaluation at these positions (an
// energy request) reproduces them.
template <bool EV, int B, bool PF, int KB, bool ONE, int SH>
__device__ __forceinline__ int lj_loop_filter(const uint32_t* lst, int nn, uint32_t* pout, float rcd2,
                                              const float4* pbase, float4 pi, const float4* s_shift,
                                              const float* s_axis, int ti, int nt, const float* s_eps24,
                                              const float* s_sig2, float rc2, KahanF& fx, KahanF& fy, KahanF& fz,
                                              PairAcc& acc, uint32_t pad) {
  constexpr int P = B * KB;  // kept entries per compensated add
  const float e24_0 = s_eps24[0], sig2_0 = s_sig2[0];
  uint32_t wn[B];
  if (PF) {
#pragma unroll
    for (int q = 0; q < B; ++q) wn[q] = nn > 0 ? __ldg(lst + (size_t)q * 32) : 0u;
  }
  PairAcc g = {0, 0, 0, acc.pe, acc.v0, acc.v1, acc.v2, acc.v3, acc.v4, acc.v5};
  int pc = 0;
  for (int k = 0; k < nn; k += B) {
    uint32_t w[B];
    if (PF) {
#pragma unroll
      for (int q = 0; q < B; ++q) w[q] = wn[q];
      if (k + B < nn) {
#pragma unroll
        for (int q = 0; q < B; ++q) wn[q] = __ldg(lst + (size_t)(k + B + q) * 32);
      }
    } else {
#pragma unroll
      for (int q = 0; q < B; ++q) w[q] = __ldg(lst + (size_t)(k + q) * 32);
    }
    float4 pj[B];
#pragma unroll
    for (int q = 0; q < B; ++q) pj[q] = __ldg(pbase + (w[q] & kIdxMask));
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const float3 sh = entry_shift<SH>(w[q], s_shift, s_axis);
      float dx, dy, dz;
      if (pair_r2(pi, sh, pj[q], dx, dy, dz) < rcd2) {
        float e24 = e24_0, sig2 = sig2_0;
        if (!ONE) {
          const int pidx = ti * nt + w_type(w_bits(pj[q].w));
          e24 = s_eps24[pidx];
          sig2 = s_sig2[pidx];
        }
        lj_pair<EV>(g, pi, sh, pj[q], rc2, e24, sig2);
        pout[(size_t)pc * 32] = w[q];
        if (++pc % P == 0) {
          fx.add(g.fx);
          fy.add(g.fy);
          fz.add(g.fz);
          g.fx = g.fy = g.fz = 0.0f;
        }
      }
    }
  }
  // the pruned list's padding: its entries, and the compensated adds of the
  // batches they complete
  const int padded = (pc + kPrunePad - 1) & ~(kPrunePad - 1);
  for (int k = pc; k < padded; ++k) pout[(size_t)k * 32] = pad;
  for (int f = pc / P; f < (padded + P - 1) / P; ++f) {
    fx.add(g.fx);
    fy.add(g.fy);
    fz.add(g.fz);
    g.fx = g.fy = g.fz = 0.0f;
  }
  acc.pe = g.pe;
  acc.v0 = g.v0;
  acc.v1 = g.v1;
  acc.v2 = g.v2;
  acc.v3 = g.v3;
  acc.v4 = g.v4;
  acc.v5 = g.v5;
  return pc;
}

// Harmonic angle (angle.cu:17-80) on (ri, rj = vertex, rk): force on the
// member `role` (0: i, 1: j, 2: k), selected without branching so that lanes
// in different roles follow one path.  EV: a third of the energy per member,
// the angle's virial carried by the vertex.
template <bool EV>
__device__ __forceinline__ void angle_term(float4 ri, float4 rj, float4 rk, int role, float kt, float th0, int G,
                                           float h, float inv_h, float dL, KahanF& fx, KahanF& fy, KahanF& fz,
                                           float& pe, float* bv) {
  const float3 dij = bonded_dr(ri, rj, G, h, inv_h, dL);
  const float3 dkj = bonded_dr(rk, rj, G, h, inv_h, dL);
  const float rij2 = dij.x * dij.x + dij.y * dij.y + dij.z * dij.z;
  const float rkj2 = dkj.x * dkj.x + dkj.y * dkj.y + dkj.z * dkj.z;
  const float rij_inv = rsqrtf(rij2), rkj_inv = rsqrtf(rkj2);
  float cs = (dij.x * dkj.x + dij.y * dkj.y + dij.z * dkj.z) * rij_inv * rkj_inv;
  cs = fminf(fmaxf(cs, -1.0f), 1.0f);
  const float dth = acosf(cs) - th0;
  const float sn = fmaxf(sqrtf(1.0f - cs * cs), 1e-6f);
  const float pref = 2.0f * kt * dth * __fdividef(1.0f, sn);
  const float rr = rij_inv * rkj_inv, i2 = rij_inv * rij_inv, k2 = rkj_inv * rkj_inv;
  // explicit roundings: the products feed the force sums in both flavours
  const float ci2 = __fmul_rn(cs, i2), ck2 = __fmul_rn(cs, k2);
  const float fix = __fmul_rn(pref, fmaf(dkj.x, rr, -__fmul_rn(ci2, dij.x)));
  const float fiy = __fmul_rn(pref, fmaf(dkj.y, rr, -__fmul_rn(ci2, dij.y)));
  const float fiz = __fmul_rn(pref, fmaf(dkj.z, rr, -__fmul_rn(ci2, dij.z)));
  const float fkx = __fmul_rn(pref, fmaf(dij.x, rr, -__fmul_rn(ck2, dkj.x)));
  const float fky = __fmul_rn(pref, fmaf(dij.y, rr, -__fmul_rn(ck2, dkj.y)));
  const float fkz = __fmul_rn(pref, fmaf(dij.z, rr, -__fmul_rn(ck2, dkj.z)));
  fx.add(role == 0 ? fix : (role == 2 ? fkx : -(fix + fkx)));
  fy.add(role == 0 ? fiy : (role == 2 ? fky : -(fiy + fky)));
  fz.add(role == 0 ? fiz : (role == 2 ? fkz : -(fiz + fkz)));
  if (EV) {
    if (role == 1) {
      bv[0] += fix * dij.x + fkx * dkj.x;
      bv[1] += fix * dij.y + fkx * dkj.y;
      bv[2] += fix * dij.z + fkx * dkj.z;
      bv[3] += fiy * dij.y + fky * dkj.y;
      bv[4] += fiy * dij.z + fky * dkj.z;
      bv[5] += fiz * dij.z + fkz * dkj.z;
    }
    pe += kt * dth * dth * (1.0f / 3.0f);
  }
}

// Forces of one chunk (block-uniform: every thread of the block calls it
// with the same chunk).  Two instantiations: with energies / virial (thermo
// steps, NPT, host requests) and without (all other steps); a chunk is
// computed by the one that matches its replica's need this step and the
// other returns at once.  skip_rebuilt: leave replicas that rebuild their
// list this step to the work-list launch that follows their rebuild.
// LISTED: the work-list launch itself (replicas rebuilt or re-filtered this
// step), which walks the rc + skin list and, where the replica keeps a
// pruned list, writes it (the filter) and its displacement reference.
// Bonded terms of the atom in slot s, gathered: its bonds and angles
// first, first + stride, ... (lanes that share an atom split them; one lane
// per atom takes all with first = 0, stride = 1).
template <bool EV>
__device__ __forceinline__ void bonded_terms(const Dev& d, const Rep& R, int s, const float4* pbase, float4 pi, int G,
                                             float h, float inv_h, float dL, int first, int stride, KahanF& fx,
                                             KahanF& fy, KahanF& fz, float& pe, float* bv, int& status) {
  const int tc = d.tcnt[s];
  const int nbd = tc & 0xFF, nang = tc >> 8;
  // FENE + WCA (fene.cu:18-73), gathered: this atom's force; the bond's
  // energy is split half per atom and its virial carried by the first atom.
  const uint32_t* bl = d.bnd + (size_t)s * kMaxBondsPerAtom;
  for (int b = first; b < nbd; b += stride) {
    const uint32_t bw = bl[b];
    const int bt = (bw >> 26) & 0xF;
    const float4 pj = pbase[bw & kSlotMask26];
    const float3 dr = bonded_dr(pi, pj, G, h, inv_h, dL);
    const float r2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
    const float kf = R.fene[4 * bt], R02 = R.fene[4 * bt + 1], eps = R.fene[4 * bt + 2], sig2 = R.fene[4 * bt + 3];
    if (r2 >= R02 * 0.9999f) status |= kStatusFeneStretch;
    const float r2s = fminf(fmaxf(r2, 1e-6f), R02 * 0.9999f);
    float ff = -kf * R02 * __fdividef(1.0f, R02 - r2s);
    float wpe = 0.0f;
    if (r2s < sig2 * 1.2599210498948732f) {
      const float r2inv = __fdividef(1.0f, r2s);
      const float sr2 = sig2 * r2inv;
      const float sr6 = sr2 * sr2 * sr2;
      ff = fmaf(24.0f * eps * r2inv * sr6, 2.0f * sr6 - 1.0f, ff);
      if (EV) wpe = 4.0f * eps * sr6 * (sr6 - 1.0f) + eps;
    }
    fx.add(__fmul_rn(ff, dr.x));
    fy.add(__fmul_rn(ff, dr.y));
    fz.add(__fmul_rn(ff, dr.z));
    if (EV) {
      pe += 0.5f * (-0.5f * kf * R02 * log1pf(-r2s / R02) + wpe);
      if ((bw >> 30) & 1) {
        bv[0] = fmaf(ff * dr.x, dr.x, bv[0]);
        bv[1] = fmaf(ff * dr.x, dr.y, bv[1]);
        bv[2] = fmaf(ff * dr.x, dr.z, bv[2]);
        bv[3] = fmaf(ff * dr.y, dr.y, bv[3]);
        bv[4] = fmaf(ff * dr.y, dr.z, bv[4]);
        bv[5] = fmaf(ff * dr.z, dr.z, bv[5]);
      }
    }
  }
  // Harmonic angles this atom belongs to, by role.
  const uint2* al = d.ang + (size_t)s * kMaxAnglesPerAtom;
  for (int a = first; a < nang; a += stride) {
    const uint2 aw = al[a];
    const int role = (aw.x >> 26) & 3, at = (aw.y >> 26) & 0xF;
    const float4 p1 = pbase[aw.x & kSlotMask26];
    const float4 p2 = pbase[aw.y & kSlotMask26];
    const float kt = R.angp[2 * at], th0 = R.angp[2 * at + 1];
    // members in angle order (i, j = vertex, k); the table holds the other two
    const float4 ri = role == 0 ? pi : p1;
    const float4 rj = role == 1 ? pi : (role == 0 ? p1 : p2);
    const float4 rk = role == 2 ? pi : p2;
    angle_term<EV>(ri, rj, rk, role, kt, th0, G, h, inv_h, dL, fx, fy, fz, pe, bv);
  }
}

// PF: 0 = list words loaded with the batch, 1 = the next batch's words
// loaded ahead into registers, D >= 2 = the ring of D batches (per-chunk
// kernel; the work-list kernel then loads ahead into registers).
template <bool EV, int B, int PF, int KB, bool LISTED, int SH, bool P2>
__device__ __forceinline__ void force_chunk(const Dev& d, int chunk, bool skip_rebuilt) {
  constexpr bool RING = PF >= 2 && !LISTED;
  constexpr bool PFR = PF != 0;  // register look-ahead in the loops below
  static_assert(!RING || B == 4, "the ring stages batches of 4 rows");
  const int4 ci = d.chunk_rep[chunk];
  const int r = ci.x;
  if (r < 0) return;
  const Rep& R = d.reps[r];
  if (!R.adv) return;
  if (need_ev(R) != EV) return;
  if (skip_rebuilt && R.rebuild_now) return;
  constexpr bool ev = EV;
  __shared__ float4 s_shift[SH == 0 ? kShiftCodes : 1];
  __shared__ float s_axis[5];
  __shared__ float s_eps24[kMaxTypes * kMaxTypes], s_sig2[kMaxTypes * kMaxTypes];
  const int nt = R.ntypes;
  const int G = R.G;
  const float h = R.h, inv_h = 1.0f / h;
  const float dL = (float)(R.L - (double)G * (double)h);
  for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
    s_eps24[k] = R.lj_eps24[k];
    s_sig2[k] = R.lj_sig2[k];
  }
  if (SH == 0 && threadIdx.x < kShiftCodes) {
    const int c = threadIdx.x;
    const int ax = c / 25, ay = (c / 5) % 5, az = c % 5;
    s_shift[c] = make_float4(shift_term(axis_code_e(ax), axis_code_k(ax), h, dL),
                             shift_term(axis_code_e(ay), axis_code_k(ay), h, dL),
                             shift_term(axis_code_e(az), axis_code_k(az), h, dL), 0.0f);
  }
  if (SH == 1 && threadIdx.x < 5)
    s_axis[threadIdx.x] = shift_term(axis_code_e(threadIdx.x), axis_code_k(threadIdx.x), h, dL);
  __syncthreads();
  const int local = ci.w * kChunk + threadIdx.x;
  const int base = R.slot_base;
  const int s = ci.y + threadIdx.x;
  const float rc2 = (float)(R.rc * R.rc);
  double vals[7] = {0, 0, 0, 0, 0, 0, 0};
  int status = 0;
  KahanF fx = {0, 0}, fy = {0, 0}, fz = {0, 0};
  PairAcc acc = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if constexpr (RING) {
    // the whole warp walks its tile's lists (lanes past natoms with none)
    __shared__ __align__(16) uint32_t s_ring[(kChunk / 32) * (RING ? PF : 1) * 4 * 32];
    const bool valid = local < R.natoms;
    const float4 pi = valid ? d.pos[s] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int ti = w_type(w_bits(pi.w));
    const bool keeps = R.prune_delta > 0.f;
    const int nn = !valid ? 0
                   : keeps ? (d.pcnt[s] + kPrunePad - 1) & ~(kPrunePad - 1)
                           : (d.ncnt[s] + kListPad - 1) & ~(kListPad - 1);
    const int nmax = __reduce_max_sync(0xffffffffu, nn);
    const uint32_t* tile_rows = (keeps ? d.pnbr : d.nbr) + (size_t)R.nbr_base + (size_t)(local >> 5) * R.M * 32;
    uint32_t* ring = s_ring + (threadIdx.x >> 5) * (PF * 4 * 32);
    const uint32_t pad = (uint32_t)local | kPadBits;
    if (nt == 1)
      lj_loop_ring<EV, KB, true, SH, P2, (RING ? PF : 2)>(tile_rows, ring, threadIdx.x & 31, nn, nmax, pad,
                                                          d.pos + base, pi, s_shift, s_axis, ti, nt, s_eps24, s_sig2,
                                                          rc2, fx, fy, fz, acc);
    else
      lj_loop_ring<EV, KB, false, SH, P2, (RING ? PF : 2)>(tile_rows, ring, threadIdx.x & 31, nn, nmax, pad,
                                                           d.pos + base, pi, s_shift, s_axis, ti, nt, s_eps24,
                                                           s_sig2, rc2, fx, fy, fz, acc);
  }
  if (local < R.natoms) {
    const float4 pi = d.pos[s];
    const uint32_t ui = w_bits(pi.w);
    const int ti = w_type(ui);
    static_assert(kListPad % B == 0 && kPrunePad % B == 0, "list padding must cover whole batches");
    // the pruned list when the replica keeps one (same layout and bases)
    const bool keeps = R.prune_delta > 0.f;
    const bool pruned = keeps && !LISTED;
    const size_t row = (size_t)R.nbr_base + ((size_t)(local >> 5) * R.M) * 32 + (local & 31);
    const int nn = pruned ? (d.pcnt[s] + kPrunePad - 1) & ~(kPrunePad - 1) : (d.ncnt[s] + kListPad - 1) & ~(kListPad - 1);
    const uint32_t* lst = (pruned ? d.pnbr : d.nbr) + row;
    const float4* pbase = d.pos + base;
    if (RING) {
      // the LJ sums are in already
    } else if (LISTED && keeps) {
      const float rcd = (float)(R.rc + (double)R.prune_delta);
      const uint32_t pad = (uint32_t)local | kPadBits;
      const int pc = nt == 1 ? lj_loop_filter<EV, B, PFR, KB, true, SH>(lst, nn, d.pnbr + row, rcd * rcd, pbase,
                                                                         pi, s_shift, s_axis, ti, nt, s_eps24, s_sig2,
                                                                         rc2, fx, fy, fz, acc, pad)
                             : lj_loop_filter<EV, B, PFR, KB, false, SH>(lst, nn, d.pnbr + row, rcd * rcd, pbase,
                                                                          pi, s_shift, s_axis, ti, nt, s_eps24,
                                                                          s_sig2, rc2, fx, fy, fz, acc, pad);
      d.pcnt[s] = pc;
      const float4 q = d.ref[s];
      d.ref[s] = make_float4(pi.x, pi.y, pi.z, q.w);
    } else if (nt == 1) {
      // one type (the Kremer-Grest melt): the pair parameters are loop constants
      lj_loop<EV, B, PFR, KB, true, SH, P2>(lst, nn, pbase, pi, s_shift, s_axis, ti, nt, s_eps24, s_sig2, rc2, fx,
                                             fy, fz, acc);
    } else {
      lj_loop<EV, B, PFR, KB, false, SH, P2>(lst, nn, pbase, pi, s_shift, s_axis, ti, nt, s_eps24, s_sig2, rc2, fx,
                                              fy, fz, acc);
    }
    float pe = acc.pe;
    // LJ virial: 1/2 f (x) r per half pair (lj.cu:56-61).
    float bv[6] = {0.5f * acc.v0, 0.5f * acc.v1, 0.5f * acc.v2, 0.5f * acc.v3, 0.5f * acc.v4, 0.5f * acc.v5};
    if (R.fcap > 0.0) {  // push-off caps the non-bonded force only
      float lx = fx.s - fx.c, ly = fy.s - fy.c, lz = fz.s - fz.c;
      const float m2 = lx * lx + ly * ly + lz * lz;
      const float cap = (float)R.fcap;
      if (m2 > cap * cap) {
        const float sc = cap * rsqrtf(m2);
        lx *= sc;
        ly *= sc;
        lz *= sc;
      }
      fx = {lx, 0.0f};
      fy = {ly, 0.0f};
      fz = {lz, 0.0f};
    }
    bonded_terms<EV>(d, R, s, pbase, pi, G, h, inv_h, dL, 0, 1, fx, fy, fz, pe, bv, status);
    const float ox = fx.s - fx.c, oy = fy.s - fy.c, oz = fz.s - fz.c;
    if (!isfinite(ox + oy + oz + pe)) status |= kStatusNonFinite;
    d.force[s] = make_float4(ox, oy, oz, pe);
    if (ev) {
      vals[0] = pe;
      for (int c = 0; c < 6; ++c) vals[1 + c] = bv[c];
    }
  }
  status = __syncthreads_or(status);
  if (threadIdx.x == 0 && status) atomicOr((int*)&d.reps[r].status, status);
  if (EV) block_partials<kChunk>(vals, 7, d.part + chunk, d.part_stride);
}

// The list filter alone: the entries of the atom's rc + skin list (nn
// padded entries) within rc + prune_delta, in list order, padded to whole
// force batches; returns their count.  The filter test rounds as pair_r2.
template <int SH>
__device__ __forceinline__ int filter_list(const uint32_t* lst, int nn, uint32_t* pout, float rcd2,
                                           const float4* pbase, float4 pi, const float4* s_shift, const float* s_axis,
                                           uint32_t pad) {
  int pc = 0;
  for (int k = 0; k < nn; k += kListPad) {
    uint32_t w[kListPad];
    float4 pj[kListPad];
#pragma unroll
    for (int q = 0; q < kListPad; ++q) w[q] = __ldg(lst + (size_t)(k + q) * 32);
#pragma unroll
    for (int q = 0; q < kListPad; ++q) pj[q] = __ldg(pbase + (w[q] & kIdxMask));
#pragma unroll
    for (int q = 0; q < kListPad; ++q) {
      float dx, dy, dz;
      if (pair_r2(pi, entry_shift<SH>(w[q], s_shift, s_axis), pj[q], dx, dy, dz) < rcd2)
        pout[(size_t)(pc++) * 32] = w[q];
    }
  }
  const int padded = (pc + kPrunePad - 1) & ~(kPrunePad - 1);
  for (int k = pc; k < padded; ++k) pout[(size_t)k * 32] = pad;
  return pc;
}

// Compensated sums of the lanes that share an atom (lane group g = lane /
// APW, APW = 32 / LPA atoms per warp), combined into group 0's lane by a
// shuffle tree in a fixed order: each step adds the partner's sum and then
// its compensation.
template <int LPA>
__device__ __forceinline__ void lanes_combine(KahanF& k) {
#pragma unroll
  for (int off = 16; off >= 32 / LPA; off >>= 1) {
    const float ps = __shfl_down_sync(0xffffffffu, k.s, off);
    const float pc = __shfl_down_sync(0xffffffffu, k.c, off);
    k.add(ps);
    k.add(-pc);
  }
}
template <int LPA>
__device__ __forceinline__ void lanes_sum(float& v) {
#pragma unroll
  for (int off = 16; off >= 32 / LPA; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
}

// Lanes per atom (LPA = 2 or 4): LPA lanes of a warp share one atom, 32 / LPA
// atoms per warp with an atom's lanes 32 / LPA apart, and the chunk's atoms
// are taken in LPA passes of 128 / LPA.  Lane group g walks the list batches
// g, g + LPA, ... (a load of one batch row reads 32 / LPA neighboring atoms'
// words: whole 32-byte sectors for LPA <= 4), then its share of the bonded
// terms; the groups' compensated sums are combined in group 0.  A replica
// whose pruned list is due (LISTED) first has it filtered, one thread per
// atom, and the lanes then walk the new pruned list as the per-chunk kernel
// will at the next steps, so a re-evaluation reproduces the forces.
template <bool EV, int B, bool PF, int KB, bool LISTED, int SH, bool P2, int LPA>
__device__ __forceinline__ void force_chunk_lanes(const Dev& d, int chunk, bool skip_rebuilt) {
  static_assert(LPA == 2 || LPA == 4, "two or four lanes per atom");
  constexpr int APW = 32 / LPA;
  const int4 ci = d.chunk_rep[chunk];
  const int r = ci.x;
  if (r < 0) return;
  const Rep& R = d.reps[r];
  if (!R.adv) return;
  if (need_ev(R) != EV) return;
  if (skip_rebuilt && R.rebuild_now) return;
  __shared__ float4 s_shift[SH == 0 ? kShiftCodes : 1];
  __shared__ float s_axis[5];
  __shared__ float s_eps24[kMaxTypes * kMaxTypes], s_sig2[kMaxTypes * kMaxTypes];
  const int nt = R.ntypes;
  const int G = R.G;
  const float h = R.h, inv_h = 1.0f / h;
  const float dL = (float)(R.L - (double)G * (double)h);
  for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
    s_eps24[k] = R.lj_eps24[k];
    s_sig2[k] = R.lj_sig2[k];
  }
  if (SH == 0 && threadIdx.x < kShiftCodes) {
    const int c = threadIdx.x;
    const int ax = c / 25, ay = (c / 5) % 5, az = c % 5;
    s_shift[c] = make_float4(shift_term(axis_code_e(ax), axis_code_k(ax), h, dL),
                             shift_term(axis_code_e(ay), axis_code_k(ay), h, dL),
                             shift_term(axis_code_e(az), axis_code_k(az), h, dL), 0.0f);
  }
  if (SH == 1 && threadIdx.x < 5)
    s_axis[threadIdx.x] = shift_term(axis_code_e(threadIdx.x), axis_code_k(threadIdx.x), h, dL);
  __syncthreads();
  const int base = R.slot_base;
  const float4* pbase = d.pos + base;
  const bool keeps = R.prune_delta > 0.f;
  if (LISTED && keeps) {
    const int local = ci.w * kChunk + threadIdx.x;
    if (local < R.natoms) {
      const int s = ci.y + threadIdx.x;
      const float4 pi = d.pos[s];
      const float rcd = (float)(R.rc + (double)R.prune_delta);
      const size_t row = (size_t)R.nbr_base + ((size_t)(local >> 5) * R.M) * 32 + (local & 31);
      const int nn = (d.ncnt[s] + kListPad - 1) & ~(kListPad - 1);
      const uint32_t pad = (uint32_t)local | kPadBits;
      d.pcnt[s] = filter_list<SH>(d.nbr + row, nn, d.pnbr + row, rcd * rcd, pbase, pi, s_shift, s_axis, pad);
      const float4 q = d.ref[s];
      d.ref[s] = make_float4(pi.x, pi.y, pi.z, q.w);
    }
    __syncthreads();  // the block's pruned lists are written
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane / APW;
  const float rc2 = (float)(R.rc * R.rc);
  double vals[7] = {0, 0, 0, 0, 0, 0, 0};
  int status = 0;
  static_assert(kListPad % B == 0 && kPrunePad % B == 0, "list padding must cover whole batches");
#pragma unroll 1
  for (int pass = 0; pass < LPA; ++pass) {
    const int at = pass * (kChunk / LPA) + warp * APW + lane % APW;
    const int local = ci.w * kChunk + at;
    const int s = ci.y + at;
    const bool valid = local < R.natoms;
    KahanF fx = {0, 0}, fy = {0, 0}, fz = {0, 0};
    PairAcc acc = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
      pi = d.pos[s];
      const int ti = w_type(w_bits(pi.w));
      const size_t row = (size_t)R.nbr_base + ((size_t)(local >> 5) * R.M) * 32 + (local & 31);
      const int nn = keeps ? (d.pcnt[s] + kPrunePad - 1) & ~(kPrunePad - 1)
                           : (d.ncnt[s] + kListPad - 1) & ~(kListPad - 1);
      const uint32_t* lst = (keeps ? d.pnbr : d.nbr) + row;
      if (nt == 1)
        lj_loop<EV, B, PF, KB, true, SH, P2, LPA>(lst, nn, pbase, pi, s_shift, s_axis, ti, nt, s_eps24, s_sig2, rc2,
                                                  fx, fy, fz, acc, g * B);
      else
        lj_loop<EV, B, PF, KB, false, SH, P2, LPA>(lst, nn, pbase, pi, s_shift, s_axis, ti, nt, s_eps24, s_sig2,
                                                   rc2, fx, fy, fz, acc, g * B);
    }
    if (R.fcap > 0.0) {  // push-off caps the non-bonded force total (replica-uniform branch)
      lanes_combine<LPA>(fx);
      lanes_combine<LPA>(fy);
      lanes_combine<LPA>(fz);
      float lx = fx.s - fx.c, ly = fy.s - fy.c, lz = fz.s - fz.c;
      const float m2 = lx * lx + ly * ly + lz * lz;
      const float cap = (float)R.fcap;
      if (m2 > cap * cap) {
        const float sc = cap * rsqrtf(m2);
        lx *= sc;
        ly *= sc;
        lz *= sc;
      }
      const bool own = g == 0;
      fx = {own ? lx : 0.0f, 0.0f};
      fy = {own ? ly : 0.0f, 0.0f};
      fz = {own ? lz : 0.0f, 0.0f};
    }
    float pe = acc.pe;
    float bv[6] = {0.5f * acc.v0, 0.5f * acc.v1, 0.5f * acc.v2, 0.5f * acc.v3, 0.5f * acc.v4, 0.5f * acc.v5};
    if (valid) bonded_terms<EV>(d, R, s, pbase, pi, G, h, inv_h, dL, g, LPA, fx, fy, fz, pe, bv, status);
    lanes_combine<LPA>(fx);
    lanes_combine<LPA>(fy);
    lanes_combine<LPA>(fz);
    if (EV) {
      lanes_sum<LPA>(pe);
#pragma unroll
      for (int c = 0; c < 6; ++c) lanes_sum<LPA>(bv[c]);
    }
    if (valid && g == 0) {
      const float ox = fx.s - fx.c, oy = fy.s - fy.c, oz = fz.s - fz.c;
      if (!isfinite(ox + oy + oz + pe)) status |= kStatusNonFinite;
      d.force[s] = make_float4(ox, oy, oz, pe);
      if (EV) {
        vals[0] += pe;
        for (int c = 0; c < 6; ++c) vals[1 + c] += bv[c];
      }
    }
  }
  status = __syncthreads_or(status);
  if (threadIdx.x == 0 && status) atomicOr((int*)&d.reps[r].status, status);
  if (EV) block_partials<kChunk>(vals, 7, d.part + chunk, d.part_stride);
}

// One block per chunk of the batch.
template <bool EV, int B, int MINB, int PF, int KB, int SH, bool P2, int LPA>
__global__ void __launch_bounds__(kChunk, MINB) k_force(Dev d, int skip_rebuilt) {
  count_launch(d, EV ? kKForceEv : kKForce);
  if constexpr (LPA == 1)
    force_chunk<EV, B, PF, KB, false, SH, P2>(d, blockIdx.x, skip_rebuilt != 0);
  else
    force_chunk_lanes<EV, B, (PF != 0), KB, false, SH, P2, LPA>(d, blockIdx.x, skip_rebuilt != 0);
}

// The chunks of the replicas on the rebuild work list (a resident grid
// striding over them), launched after their rebuild while the other
// replicas' forces run beside it; it also writes their pruned lists.
template <bool EV, int B, int MINB, int PF, int KB, int SH, bool P2, int LPA>
__global__ void __launch_bounds__(kChunk, MINB) k_force_rb(Dev d) {
  count_launch(d, EV ? kKForceEv : kKForce);
  const int n = rb_count(d);
  const int* off = rb_off(d, 3);
  const int total = n > 0 ? off[n] : 0;
  RbCursor cur(off, n, blockIdx.x);
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    cur.seek(item);
    __syncthreads();  // the previous item's shared tables are no longer read
    const Rep& R = d.reps[rb_rep(d, cur.i)];
    if constexpr (LPA == 1)
      force_chunk<EV, B, PF, KB, true, SH, P2>(d, R.chunk_base + (item - cur.lo), false);
    else
      force_chunk_lanes<EV, B, (PF != 0), KB, true, SH, P2, LPA>(d, R.chunk_base + (item - cur.lo), false);
  }
}

// ---------------------------------------------------------------- pruned list
// Filter of the listed replicas' lists (after a rebuild, or when the
// displacement since the last filter reached prune_delta / 2): the entries
// of the rc + skin list within rc + prune_delta at the current positions, in
// list order, padded like the full list; the positions become the new
// displacement reference.  Replicas without a pruned list are skipped.
__global__ void __launch_bounds__(kChunk) k_prune(Dev d) {
  count_launch(d, kKPlan);
  const int n = rb_count(d);
  const int* off = rb_off(d, 3);
  const int total = n > 0 ? off[n] : 0;
  __shared__ float4 s_shift[kShiftCodes];
  RbCursor cur(off, n, blockIdx.x);
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    cur.seek(item);
    __syncthreads();  // the previous item's shift table is no longer read
    const Rep& R = d.reps[rb_rep(d, cur.i)];
    if (R.prune_delta <= 0.f) continue;  // block-uniform
    const int G = R.G;
    const float h = R.h;
    const float dL = (float)(R.L - (double)G * (double)h);
    if (threadIdx.x < kShiftCodes) {
      const int c = threadIdx.x;
      const int ax = c / 25, ay = (c / 5) % 5, az = c % 5;
      s_shift[c] = make_float4(shift_term(axis_code_e(ax), axis_code_k(ax), h, dL),
                               shift_term(axis_code_e(ay), axis_code_k(ay), h, dL),
                               shift_term(axis_code_e(az), axis_code_k(az), h, dL), 0.0f);
    }
    __syncthreads();
    const int local = (item - cur.lo) * kChunk + threadIdx.x;
    if (local >= R.natoms) continue;
    const int base = R.slot_base, s = base + local;
    const float4 pi = d.pos[s];
    const float rcd = (float)(R.rc + (double)R.prune_delta);
    const float rcd2 = rcd * rcd;
    const size_t row0 = (size_t)R.nbr_base + ((size_t)(local >> 5) * R.M) * 32 + (local & 31);
    const uint32_t* in = d.nbr + row0;
    uint32_t* out = d.pnbr + row0;
    const float4* pbase = d.pos + base;
    // batches of kListPad entries (the full list's padding lies beyond
    // rc + prune_delta and drops out): all words, then all gathers, then
    // the tests, so the loads of a batch are in flight together
    const int nn = (d.ncnt[s] + kListPad - 1) & ~(kListPad - 1);
    int cnt = 0;
    for (int k = 0; k < nn; k += kListPad) {
      uint32_t w[kListPad];
      float4 pj[kListPad];
#pragma unroll
      for (int q = 0; q < kListPad; ++q) w[q] = __ldg(in + (size_t)(k + q) * 32);
#pragma unroll
      for (int q = 0; q < kListPad; ++q) pj[q] = __ldg(pbase + (w[q] & kIdxMask));
#pragma unroll
      for (int q = 0; q < kListPad; ++q) {
        const float3 sh = entry_shift<0>(w[q], s_shift, nullptr);
        const float dx = (pi.x - pj[q].x) - sh.x, dy = (pi.y - pj[q].y) - sh.y, dz = (pi.z - pj[q].z) - sh.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < rcd2) out[(size_t)(cnt++) * 32] = w[q];
      }
    }
    const int padded = (cnt + kPrunePad - 1) & ~(kPrunePad - 1);
    for (int k = cnt; k < padded; ++k) out[(size_t)k * 32] = (uint32_t)local | kPadBits;
    d.pcnt[s] = cnt;
    const float4 q = d.ref[s];
    d.ref[s] = make_float4(pi.x, pi.y, pi.z, q.w);
  }
}

void launch_prune(const Dev& d, cudaStream_t st);

// ---------------------------------------------------------------- pair tables
// Tabulated pair potential (force/table.cu:60-110 semantics): for listed
// pairs within rc whose type pair has a table, r is clamped to the grid,
// the force column (applied as F/r) and the energy are interpolated
// linearly between the two grid points around r; half the energy and half
// the virial per side.  A second pass over the list, run after the force
// kernel for replicas with tables only; explicit roundings keep the energy
// flavour's forces identical to the plain one's.
template <bool EV>
__global__ void __launch_bounds__(kChunk) k_table(Dev d, int sel) {
  count_launch(d, kKTable);
  const int chunk = blockIdx.x;
  const int4 ci = d.chunk_rep[chunk];
  const int r = ci.x;
  if (r < 0) return;
  const Rep& R = d.reps[r];
  if (!R.adv || R.ntables == 0 || need_ev(R) != EV) return;
  if ((sel == 1 && R.rebuild_now) || (sel == 2 && !R.rebuild_now)) return;
  __shared__ float4 s_shift[kShiftCodes];
  const int G = R.G;
  const float h = R.h;
  const float dL = (float)(R.L - (double)G * (double)h);
  if (threadIdx.x < kShiftCodes) {
    const int c = threadIdx.x;
    const int ax = c / 25, ay = (c / 5) % 5, az = c % 5;
    s_shift[c] = make_float4(shift_term(axis_code_e(ax), axis_code_k(ax), h, dL),
                             shift_term(axis_code_e(ay), axis_code_k(ay), h, dL),
                             shift_term(axis_code_e(az), axis_code_k(az), h, dL), 0.0f);
  }
  __syncthreads();
  const int local = ci.w * kChunk + threadIdx.x;
  const int s = ci.y + threadIdx.x;
  const float rc2 = (float)(R.rc * R.rc);
  const int nt = R.ntypes;
  double vals[7] = {0, 0, 0, 0, 0, 0, 0};
  if (local < R.natoms) {
    const float4 pi = d.pos[s];
    const int ti = w_type(w_bits(pi.w));
    // the pruned list when the replica keeps one (same layout and bases)
    const bool pruned = R.prune_delta > 0.f;
    const int nn = pruned ? (d.pcnt[s] + kPrunePad - 1) & ~(kPrunePad - 1) : (d.ncnt[s] + kListPad - 1) & ~(kListPad - 1);
    const uint32_t* lst = (pruned ? d.pnbr : d.nbr) + R.nbr_base + ((size_t)(local >> 5) * R.M) * 32 + (local & 31);
    const float4* pbase = d.pos + R.slot_base;
    float fx = 0, fy = 0, fz = 0, pe = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
    for (int k = 0; k < nn; ++k) {
      const uint32_t w = __ldg(lst + (size_t)k * 32);
      const float4 pj = __ldg(pbase + (w & kIdxMask));
      const float3 sh = entry_shift<0>(w, s_shift, nullptr);
      const float dx = __fsub_rn(__fsub_rn(pi.x, pj.x), sh.x);
      const float dy = __fsub_rn(__fsub_rn(pi.y, pj.y), sh.y);
      const float dz = __fsub_rn(__fsub_rn(pi.z, pj.z), sh.z);
      const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      const int tid = R.table_of[ti * nt + w_type(w_bits(pj.w))];
      if (!(r2 < rc2 && r2 > 1e-10f) || tid < 0) continue;
      const float rmin = R.tab_rmin[tid], rmax = R.tab_rmax[tid], dr = R.tab_dr[tid], inv_dr = R.tab_inv_dr[tid];
      const int np = R.tab_n[tid];
      const float rr = fminf(fmaxf(__fsqrt_rn(r2), rmin), rmax);
      int idx = (int)__fmul_rn(__fsub_rn(rr, rmin), inv_dr);
      idx = max(0, min(idx, np - 2));
      const float t = __fmul_rn(__fsub_rn(rr, __fadd_rn(rmin, __fmul_rn((float)idx, dr))), inv_dr);
      const float2 p0 = __ldg(d.tab + R.tab_off[tid] + idx), p1 = __ldg(d.tab + R.tab_off[tid] + idx + 1);
      const float fs = __fadd_rn(p0.x, __fmul_rn(t, __fsub_rn(p1.x, p0.x)));
      const float fxij = __fmul_rn(fs, dx), fyij = __fmul_rn(fs, dy), fzij = __fmul_rn(fs, dz);
      fx = __fadd_rn(fx, fxij);
      fy = __fadd_rn(fy, fyij);
      fz = __fadd_rn(fz, fzij);
      if (EV) {
        const float e = __fadd_rn(p0.y, __fmul_rn(t, __fsub_rn(p1.y, p0.y)));
        pe += 0.5f * e;
        v0 += 0.5f * fxij * dx;
        v1 += 0.5f * fxij * dy;
        v2 += 0.5f * fxij * dz;
        v3 += 0.5f * fyij * dy;
        v4 += 0.5f * fyij * dz;
        v5 += 0.5f * fzij * dz;
      }
    }
    float4 f = d.force[s];
    f.x = __fadd_rn(f.x, fx);
    f.y = __fadd_rn(f.y, fy);
    f.z = __fadd_rn(f.z, fz);
    if (EV) f.w += pe;
    d.force[s] = f;
    if (EV) {
      vals[0] = pe;
      vals[1] = v0;
      vals[2] = v1;
      vals[3] = v2;
      vals[4] = v3;
      vals[5] = v4;
      vals[6] = v5;
    }
  }
  if (EV) {
    __shared__ double s_add[7];
    block_partials<kChunk>(vals, 7, s_add, 1);
    __syncthreads();
    if (threadIdx.x < 7) d.part[threadIdx.x * d.part_stride + chunk] += s_add[threadIdx.x];
  }
}

void launch_table(const Dev& d, int nchunks, bool ev, int sel, cudaStream_t st) {
  if (ev)
    k_table<true><<<nchunks, kChunk, 0, st>>>(d, sel);
  else
    k_table<false><<<nchunks, kChunk, 0, st>>>(d, sel);
}

// ---------------------------------------------------------------- post-force
__global__ void __launch_bounds__(kChunk, 7) k_post(Dev d, int kick) {
  count_launch(d, kKPost);
  const int chunk = blockIdx.x;
  const int4 ci = d.chunk_rep[chunk];
  if (ci.x < 0) return;
  const int s = ci.y + threadIdx.x;
  const bool have = (int)threadIdx.x < ci.z;
  float4 v = make_float4(0, 0, 0, 1), f = make_float4(0, 0, 0, 0);
  if (have) {
    v = d.vel[s];
    f = d.force[s];
  }
  Rep& R = d.reps[ci.x];
  if (!R.adv || (kick == 1 && R.defer)) return;
  double vals[7] = {0, 0, 0, 0, 0, 0, 0};
  if (have) {
    if (kick == 1) {
      const double dt = (R.mode == kModePushoff) ? R.push_dt : R.dt;
      const float hm = (float)(0.5 * dt) * v.w;
      v.x = fmaf(hm, f.x, v.x);
      v.y = fmaf(hm, f.y, v.y);
      v.z = fmaf(hm, f.z, v.z);
      d.vel[s] = v;
    }
    const double m = 1.0 / (double)v.w;
    const double vx = v.x, vy = v.y, vz = v.z;
    vals[0] = m * vx * vx;
    vals[1] = m * vx * vy;
    vals[2] = m * vx * vz;
    vals[3] = m * vy * vy;
    vals[4] = m * vy * vz;
    vals[5] = m * vz * vz;
  }
  block_partials<kChunk>(vals, 6, d.part + 7 * d.part_stride + chunk, d.part_stride);
}

// One pressure-tensor sample into a replica's multiple-tau correlator, by
// one warp (lanes = lags).  Follows correlator.cu:33-92: each level stores
// the sample at its insert position, adds sample x (sample `lag` positions
// back) for the lags 0 .. insert position (the reference counts lags from
// the insert position, not from the samples held), and passes the average
// of every kAcfPoints samples to the next level.  Products and sums are
// rounded separately (no contraction), so the sums are reproducible by a
// plain FP64 restatement.
__device__ void acf_push(double* st, const double* sample_in) {
  const int lane = threadIdx.x & 31;
  double smp[kAcfComps];
  for (int c = 0; c < kAcfComps; ++c) smp[c] = sample_in[c];
  for (int level = 0; level < kAcfLevels; ++level) {
    const int idx = (int)st[kAcfIdx + level];
    double* buf = st + kAcfBuf + level * kAcfPoints * kAcfComps;
    if (lane == 0)
      for (int c = 0; c < kAcfComps; ++c) buf[idx * kAcfComps + c] = smp[c];
    __syncwarp();
    const int nstored = min(idx + 1, kAcfPoints);
    if (lane < nstored) {
      const int older = (idx - lane + kAcfPoints) % kAcfPoints;
      double* corr = st + kAcfCorr + (level * kAcfPoints + lane) * kAcfComps;
      for (int c = 0; c < kAcfComps; ++c) corr[c] = __dadd_rn(corr[c], __dmul_rn(smp[c], buf[older * kAcfComps + c]));
      st[kAcfCnt + level * kAcfPoints + lane] += 1.0;
    }
    int carry = 0;
    if (lane == 0) {
      st[kAcfIdx + level] = (double)((idx + 1) % kAcfPoints);
      double* acc = st + kAcfAcc + level * kAcfComps;
      for (int c = 0; c < kAcfComps; ++c) acc[c] = __dadd_rn(acc[c], smp[c]);
      const double n = st[kAcfAccN + level] + 1.0;
      if (n >= (double)kAcfPoints) {
        for (int c = 0; c < kAcfComps; ++c) {
          smp[c] = acc[c] / (double)kAcfPoints;
          acc[c] = 0.0;
        }
        st[kAcfAccN + level] = 0.0;
        carry = 1;
      } else {
        st[kAcfAccN + level] = n;
      }
    }
    __syncwarp();
    if (!__shfl_sync(0xFFFFFFFFu, carry, 0)) break;
    for (int c = 0; c < kAcfComps; ++c) smp[c] = __shfl_sync(0xFFFFFFFFu, smp[c], 0);
  }
}

// Per-replica commit of the post-force update (one warp per replica, after
// every post-force block finished): reduce the chunk partials in chunk order
// (deterministic), store energies / virial / KE, run the post-force chain or
// barostat, and precompute the next pre-force's scalars.
__global__ void __launch_bounds__(kPostCommitThreads) k_post_commit(Dev d, int kick) {
  count_launch(d, kKCommit);
  const int r = blockIdx.x;
  if (r >= d.rb_cap) return;
  Rep& R = d.reps[r];
  if (!R.adv || (kick == 1 && R.defer)) return;
  {
    // The replica's chunk partials: thread t sums chunks t, t + T, ... in
    // order, each warp's sums are combined by a shuffle tree, and thread 0
    // adds the warp totals in warp order -- a fixed order for a given
    // replica size, so the sums are bit-reproducible and independent of the
    // rest of the batch.  (One warp for all chunks took 83 us per step on a
    // 1M-bead replica.)
    constexpr int nw = kPostCommitThreads / 32;
    __shared__ double s_red[nw][13];
    double acc[13];
    for (int q = 0; q < 13; ++q) acc[q] = 0.0;
    for (int c = threadIdx.x; c < R.nchunks; c += kPostCommitThreads) {
      const double* pp = d.part + R.chunk_base + c;
      for (int q = 0; q < 13; ++q) acc[q] += pp[q * d.part_stride];
    }
    for (int q = 0; q < 13; ++q) acc[q] = warp_sum(acc[q]);
    if ((threadIdx.x & 31) == 0)
      for (int q = 0; q < 13; ++q) s_red[threadIdx.x >> 5][q] = acc[q];
    __syncthreads();
    if (threadIdx.x >= 32) return;
    if (threadIdx.x == 0) {
      for (int q = 0; q < 13; ++q) {
        double t = s_red[0][q];
        for (int w = 1; w < nw; ++w) t += s_red[w][q];
        acc[q] = t;
      }
      if (need_ev(R)) {
        R.pe = acc[0];
        for (int q = 0; q < 6; ++q) R.vir[q] = acc[1 + q];
      }
      for (int q = 0; q < 6; ++q) R.ke[q] = acc[7 + q];
      const double ke_raw = acc[7] + acc[10] + acc[12];
      const double dt = (R.mode == kModePushoff) ? R.push_dt : R.dt;
      const int ens = (R.mode == kModePushoff) ? FMD_LANGEVIN : R.ensemble;
      if (need_ev(R)) R.ev_step = R.step;
      R.force_ev = 0;
      // the chain / barostat state is updated in a local copy and stored
      // once: in place, its arrays' stores would order every later read of
      // the record behind them
      NHScalars nh = R.nh;
      if (kick == 2) {
        // re-evaluation of the current state: reductions only
      } else if (!kick) {
        // Setup: the chain carry starts at the current KE (main.cu:376-390).
        nh.carry = 0.5 * ke_raw;
        R.pending_scale = 1.0;
      } else if (ens == FMD_NVT_NH) {
        const double kT = ramp(R, R.step, R.T0, R.T1);
        const double ke = 0.5 * ke_raw;
        const double sc = nhc_half_step(nh.xi, nh.vxi, R.chain_M, R.Q1, R.Qr, kT, R.natoms, ke, 0.5 * dt,
                                        nh.carry_dd ? nh.dd : nullptr);
        nh.scale = sc;
        nh.carry = ke * sc * sc;
        R.pending_scale = sc;
      } else if (ens == FMD_NPT_NH) {
        const double kT = ramp(R, R.step, R.T0, R.T1), Pt = ramp(R, R.step, R.P0, R.P1);
        const double vtr = R.vir[0] + R.vir[3] + R.vir[5];
        npt_chain_baro(nh, false, ke_raw, vtr, R.chain_M, R.Q1, R.Qr, R.W, 0.5 * dt, dt, R.V0, R.natoms, kT, Pt,
                       DExp(), DCbrt(), DSinh());
        R.L = nh.L;
        R.pending_scale = nh.bscale * nh.scale;
      } else {
        R.pending_scale = 1.0;
      }
      R.nh = nh;
      R.thermo_step = R.step;
      R.adv = 0;
      R.rebuild_now = 0;
      // scalars of the next pre-force, computed once here for all its blocks
      next_scalars(R);
      R.next_valid = 1;
    }
    // Stress steps: the thermo row's pressure tensor, (KE tensor (with the
    // pending thermostat scale) + virial) / V in the current box, feeds the
    // correlator (main.cu:632-666).
    __syncwarp();
    if (kick == 1 && stress_step(R)) {
      const double s2 = __dmul_rn(R.pending_scale, R.pending_scale);
      const double V = __dmul_rn(__dmul_rn(R.L, R.L), R.L);
      double smp[kAcfComps];
      for (int c = 0; c < kAcfComps; ++c) smp[c] = __dadd_rn(__dmul_rn(R.ke[c], s2), R.vir[c]) / V;
      acf_push(d.acf + (size_t)r * kAcfWords, smp);
    }
  }
}

// One trajectory frame of a replica in atom-id order: each position wrapped
// in the box of the last pre-force update, as the reference stores and dumps
// them (dump.cu:5-11, main.cu:675-679), in single precision.
__global__ void __launch_bounds__(256) k_pack_frame(Dev d, int r, float* out) {
  const Rep& R = d.reps[r];
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= R.natoms) return;
  const int s = d.slot_of[R.slot_base + id];
  const float4 p = d.pos[R.slot_base + s];
  const uint32_t u = w_bits(p.w);
  const int c[3] = {w_cx(u), w_cy(u), w_cz(u)};
  const float o[3] = {p.x, p.y, p.z};
  const double h = (double)R.h, Lp = R.Lpos;
  for (int a = 0; a < 3; ++a) {
    // the host readout's operations, rounded one by one
    double x = __dadd_rn(__dmul_rn((double)c[a], h), (double)o[a]);
    x = __dsub_rn(x, __dmul_rn(floor(x / Lp), Lp));
    out[3 * id + a] = (float)x;
  }
}

void launch_pack_frame(const Dev& d, int r, int natoms, float* out, cudaStream_t st) {
  k_pack_frame<<<(natoms + 255) / 256, 256, 0, st>>>(d, r, out);
}

// ---- full-grid rebuild kernels: one block per chunk / cell group / home
// cell of every replica (blocks of replicas that do not rebuild return at
// once).  Used when many replicas rebuild in the same step, where they beat
// the persistent work-list kernels.
__global__ void __launch_bounds__(kChunk) k_bin_g(Dev d) {
  count_launch(d, kKBin);
  const int4 ci = d.chunk_rep[blockIdx.x];
  if (ci.x < 0 || d.reps[ci.x].rebuild_now != 1) return;
  bin_chunk(d, d.reps[ci.x], ci.w);
}

__global__ void __launch_bounds__(kChunk) k_scatter_g(Dev d) {
  count_launch(d, kKScatter);
  const int4 ci = d.chunk_rep[blockIdx.x];
  if (ci.x < 0 || d.reps[ci.x].rebuild_now != 1) return;
  const Rep& R = d.reps[ci.x];
  const int local = ci.w * kChunk + threadIdx.x;
  if (local >= R.natoms) return;
  const int s = R.slot_base + local;
  const int at = atomicAdd(&d.cell_fill[R.cell_base + d.key[s]], 1);
  d.bucket[R.slot_base + at] = local;
}

__global__ void __launch_bounds__(32 * kCellGroup) k_cellsort_g(Dev d) {
  count_launch(d, kKCellsort);
  if ((int)blockIdx.y >= rb_count(d)) return;
  const Rep& R = d.reps[rb_rep(d, blockIdx.y)];
  if (R.rebuild_now != 1) return;
  const int c = blockIdx.x * kCellGroup + (threadIdx.x >> 5);
  if (c < R.P * R.P * R.P) cellsort_cell(d, R, c, threadIdx.x & 31);
}

__global__ void __launch_bounds__(kChunk) k_permute_g(Dev d) {
  count_launch(d, kKPermute);
  const int4 ci = d.chunk_rep[blockIdx.x];
  if (ci.x < 0 || d.reps[ci.x].rebuild_now != 1) return;
  permute_chunk(d, d.reps[ci.x], ci.w);
}

__global__ void __launch_bounds__(kChunk) k_topo_g(Dev d) {
  count_launch(d, kKTopo);
  const int4 ci = d.chunk_rep[blockIdx.x];
  if (ci.x < 0 || d.reps[ci.x].rebuild_now != 1) return;
  topo_chunk(d, d.reps[ci.x], ci.w);
}

__global__ void __launch_bounds__(kNbrThreads) k_neighbors_g(Dev d) {
  count_launch(d, kKNeighbors);
  if ((int)blockIdx.y >= rb_count(d)) return;
  Rep& R = d.reps[rb_rep(d, blockIdx.y)];
  if (R.rebuild_now != 1) return;
  const int G = R.G;
  if ((int)blockIdx.x >= G * G * G) return;
  neighbors_cell_ballot(d, R, blockIdx.x);
}

// ---------------------------------------------------------------- launchers
namespace {
int num_sms() {
  int dev = 0;
  FMD_CUDA(cudaGetDevice(&dev));
  static int cache[256] = {0};
  if (dev < 0 || dev >= 256) return 148;
  if (!cache[dev]) FMD_CUDA(cudaDeviceGetAttribute(&cache[dev], cudaDevAttrMultiProcessorCount, dev));
  return cache[dev];
}

// Blocks of a persistent (grid-stride) kernel: exactly the number that are
// resident at once, so no block waits for a second wave.
template <typename K>
int resident_grid(K kernel, int threads) {
  int per_sm = 0;
  FMD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
  return num_sms() * (per_sm > 0 ? per_sm : 1);
}
}  // namespace

// The pre-force update of every chunk, one block per chunk.  (A resident
// grid streaming the chunks through shared memory by asynchronous copies
// measured the same, 50.7 against 48.7 us on 64 x 30K: long-scoreboard
// stalls stayed the limit.)
void launch_pre(const Dev& d, const StepConds& c, int nchunks, cudaStream_t st) {
  k_pre<kPreAPT><<<nchunks, kChunk / kPreAPT, 0, st>>>(d, c);
}

void launch_step(const Dev& d, const StepShape& g, int* host_mode, cudaStream_t st) {
  const StepConds none{0, 0, 0, 0, 0, 0, 0};
  launch_pre(d, none, g.nchunks, st);
  k_commit<<<g.nreps, 32, 0, st>>>(d, none);
  FMD_CUDA(cudaMemcpyAsync(host_mode, d.rb + kRbMode, sizeof(int), cudaMemcpyDeviceToHost, st));
  FMD_CUDA(cudaStreamSynchronize(st));
  // the graph's kernels in one stream: the listed replicas' forces (and
  // pruned-list filters) from the work-list launch after their rebuild
  const int mode = *host_mode;
  if (mode == kRbList) launch_rebuild(d, g.nreps, g.nbr_variant, st, false);
  if (mode == kRbFull) launch_rebuild_full(d, g, st, false);
  if (mode == kRbPrune) launch_rb_plan(d, st);
  if (mode != kRbNone) {
    launch_force_rebuilt(d, false, g.force_variant, st);
    launch_force_rebuilt(d, true, g.force_variant, st);
    if (g.has_table) {
      launch_table(d, g.nchunks, false, 2, st);
      launch_table(d, g.nchunks, true, 2, st);
    }
  }
  launch_force(d, g.nchunks, false, g.force_variant, st, true);
  launch_force(d, g.nchunks, true, g.force_variant, st, true);
  if (g.has_table) {
    launch_table(d, g.nchunks, false, 1, st);
    launch_table(d, g.nchunks, true, 1, st);
  }
  k_post<<<g.nchunks, kChunk, 0, st>>>(d, 1);
  k_post_commit<<<g.nreps, kPostCommitThreads, 0, st>>>(d, 1);
}

namespace {
// Append an IF node on handle h to the graph being captured on st; its body
// is recorded on side by fn(side).
template <typename F>
void capture_if(cudaStream_t st, cudaStream_t side, cudaGraphConditionalHandle h, F&& fn) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  FMD_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) throw Error(FMD_ERR_CUDA, "conditional node outside a capture");
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  FMD_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  cudaGraph_t body = p.conditional.phGraph_out[0];
  FMD_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  fn(side);
  cudaGraph_t done;
  FMD_CUDA(cudaStreamEndCapture(side, &done));
  FMD_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
}
}  // namespace

void capture_step(const Dev& d, const StepShape& shape, cudaStream_t st, cudaStream_t side, cudaStream_t side_hi,
                  const cudaStream_t* br) {
  const int nchunks = shape.nchunks, nreps = shape.nreps, force_variant = shape.force_variant,
            nbr_variant = shape.nbr_variant;
  cudaStreamCaptureStatus cs;
  cudaGraph_t g;
  FMD_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
  StepConds c{1, 0, 0, 0, 0, 0, 0};
  FMD_CUDA(cudaGraphConditionalHandleCreate(&c.rebuild, g, 0u, cudaGraphCondAssignDefault));
  FMD_CUDA(cudaGraphConditionalHandleCreate(&c.rebuild_full, g, 0u, cudaGraphCondAssignDefault));
  FMD_CUDA(cudaGraphConditionalHandleCreate(&c.force_ev, g, 0u, cudaGraphCondAssignDefault));
  FMD_CUDA(cudaGraphConditionalHandleCreate(&c.post, g, 0u, cudaGraphCondAssignDefault));
  FMD_CUDA(cudaGraphConditionalHandleCreate(&c.prune, g, 0u, cudaGraphCondAssignDefault));
  launch_pre(d, c, nchunks, st);
  k_commit<<<nreps, 32, 0, st>>>(d, c);
  // Four parallel branches, each one conditional node: the two rebuild forms
  // (they exclude each other), each followed by the forces of the replicas
  // it rebuilt, and the two force flavours of every other replica, which so
  // run beside the rebuild instead of after it.  The rebuild bodies are
  // captured on a high-priority stream, so their blocks go first whenever
  // the force kernels free a slot.
  cudaEvent_t fork, join[4];
  FMD_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (auto& e : join) FMD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  FMD_CUDA(cudaEventRecord(fork, st));
  for (int b = 0; b < 4; ++b) FMD_CUDA(cudaStreamWaitEvent(br[b], fork, 0));
  const bool tab = shape.has_table != 0;
  capture_if(st, side_hi, c.rebuild, [&](cudaStream_t s) {
    launch_rebuild(d, nreps, nbr_variant, s, false);
    launch_force_rebuilt(d, false, force_variant, s);
    launch_force_rebuilt(d, true, force_variant, s);
    if (tab) {
      launch_table(d, nchunks, false, 2, s);
      launch_table(d, nchunks, true, 2, s);
    }
  });
  capture_if(br[0], side_hi, c.rebuild_full, [&](cudaStream_t s) {
    launch_rebuild_full(d, shape, s, false);
    launch_force_rebuilt(d, false, force_variant, s);
    launch_force_rebuilt(d, true, force_variant, s);
    if (tab) {
      launch_table(d, nchunks, false, 2, s);
      launch_table(d, nchunks, true, 2, s);
    }
  });
  // The plain flavour runs on nearly every step: a plain kernel node (its
  // blocks return at once for replicas that need the energy flavour) saves
  // the conditional node's latency.
  launch_force(d, nchunks, false, force_variant, br[1], true);
  if (tab) launch_table(d, nchunks, false, 1, br[1]);
  capture_if(br[2], side, c.force_ev, [&](cudaStream_t s) {
    launch_force(d, nchunks, true, force_variant, s, true);
    if (tab) launch_table(d, nchunks, true, 1, s);
  });
  // steps where replicas only re-filter their pruned lists skip the rebuild
  // chain: the work-list force launch filters
  capture_if(br[3], side_hi, c.prune, [&](cudaStream_t s) {
    launch_rb_plan(d, s);
    launch_force_rebuilt(d, false, force_variant, s);
    launch_force_rebuilt(d, true, force_variant, s);
    if (tab) {
      launch_table(d, nchunks, false, 2, s);
      launch_table(d, nchunks, true, 2, s);
    }
  });
  for (int b = 0; b < 4; ++b) {
    FMD_CUDA(cudaEventRecord(join[b], br[b]));
    FMD_CUDA(cudaStreamWaitEvent(st, join[b], 0));
  }
  capture_if(st, side, c.post, [&](cudaStream_t s) {
    k_post<<<nchunks, kChunk, 0, s>>>(d, 1);
    k_post_commit<<<nreps, kPostCommitThreads, 0, s>>>(d, 1);
  });
  FMD_CUDA(cudaEventDestroy(fork));
  for (auto& e : join) FMD_CUDA(cudaEventDestroy(e));
}

namespace {

int rebuild_priority() {
  static const int p = [] {
    int least = 0, greatest = 0;
    FMD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    return greatest;
  }();
  return p;
}

// Launch at the rebuild branch's priority.  Recorded in the kernel node when
// captured, it makes the block scheduler dispatch the rebuild's blocks ahead
// of the pending blocks of the force kernels running beside it.
template <typename... KArgs, typename... Args>
void launch_hi(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributePriority;
  at[0].val.priority = rebuild_priority();
  cfg.attrs = at;
  cfg.numAttrs = 1;
  FMD_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
}
}  // namespace

void launch_prune(const Dev& d, cudaStream_t st) {
  static const int g_prune = resident_grid(k_prune, kChunk);
  launch_hi(k_prune, g_prune, kChunk, st, d);
}

void launch_rb_plan(const Dev& d, cudaStream_t st) { launch_hi(k_rbplan, 1, kPlanThreads, st, d); }

void launch_prune_only(const Dev& d, cudaStream_t st) {
  launch_rb_plan(d, st);
  launch_prune(d, st);
}

void launch_rebuild_full(const Dev& d, const RebuildShape& g, cudaStream_t st, bool filter) {
  const int nr = g.nreps;
  launch_hi(k_rbplan, 1, kPlanThreads, st, d);  // work-list offsets for the forces that follow
  launch_hi(k_bin_g, g.nchunks, kChunk, st, d);
  launch_hi(k_scan, nr, kScanThreads, st, d);
  launch_hi(k_scatter_g, g.nchunks, kChunk, st, d);
  launch_hi(k_cellsort_g, dim3((g.max_cells + kCellGroup - 1) / kCellGroup, nr), 32 * kCellGroup, st, d);
  launch_hi(k_permute_g, g.nchunks, kChunk, st, d);
  launch_hi(k_topo_g, g.nchunks, kChunk, st, d);
  launch_hi(k_neighbors_g, dim3(g.max_home, nr), kNbrThreads, st, d);
  launch_hi(k_neighbors_small, dim3(8, nr), 32 * kSmallWarps, st, d);
  if (filter) launch_prune(d, st);
}

void launch_rebuild(const Dev& d, int nreps, int nbr_variant, cudaStream_t st, bool filter) {
  static const int g_bin = resident_grid(k_bin, kChunk), g_scatter = resident_grid(k_scatter, kChunk),
                   g_sort = resident_grid(k_cellsort, 32 * kCellGroup), g_perm = resident_grid(k_permute, kChunk),
                   g_topo = resident_grid(k_topo, kChunk), g_nbr0 = resident_grid(k_neighbors<0, 8>, kNbrThreads),
                   g_nbr1 = resident_grid(k_neighbors<1, 6>, kNbrThreads),
                   g_nbr2 = resident_grid(k_neighbors<0, 6>, kNbrThreads);
  launch_hi(k_rbplan, 1, kPlanThreads, st, d);
  launch_hi(k_bin, g_bin, kChunk, st, d);
  launch_hi(k_scan, nreps, kScanThreads, st, d);
  launch_hi(k_scatter, g_scatter, kChunk, st, d);
  launch_hi(k_cellsort, g_sort, 32 * kCellGroup, st, d);
  launch_hi(k_permute, g_perm, kChunk, st, d);
  launch_hi(k_topo, g_topo, kChunk, st, d);
  launch_hi(k_rbplan_home, 1, kPlanThreads, st, d, nbr_variant);
  if (nbr_variant == 1)
    launch_hi(k_neighbors<1, 6>, g_nbr1, kNbrThreads, st, d);
  else if (nbr_variant == 2)
    launch_hi(k_neighbors<0, 6>, g_nbr2, kNbrThreads, st, d);
  else
    launch_hi(k_neighbors<0, 8>, g_nbr0, kNbrThreads, st, d);
  launch_hi(k_neighbors_small, dim3(8, nreps), 32 * kSmallWarps, st, d);
  if (filter) launch_prune(d, st);
}

// Force-kernel variants (list entries per batch, blocks per SM, pipelined
// list loads, batches per compensated add); the batch's autotuner picks one.
// The energy flavour of a variant walks the list in the same batches with
// the same compensated adds, so its forces are bit-identical: energy steps
// and host re-evaluations do not perturb a trajectory.
constexpr int kForceCarveoutPct = 16;  // percent of the SM's shared-memory maximum

// The variant's two kernels: one block per chunk, and the work-list form.
// Parameters: list entries per batch, blocks per SM, next batch's list words
// loaded ahead, batches per compensated add, shift lookup (0: 125-entry 3D
// table, 1: per-axis 5-value table), pairs evaluated two at a time in packed
// FP32x2 arithmetic, lanes per atom.
template <bool EV>
void force_kernels(int variant, void (**per_chunk)(Dev, int), void (**listed)(Dev)) {
  constexpr int E = 6;  // blocks per SM of the energy flavours (more registers: up to 85)
#define FMD_FORCE_VARIANT(B, MINB, PF, KB, SH, P2, LPA)          \
  *per_chunk = k_force<EV, B, EV ? E : MINB, PF, KB, SH, P2, LPA>; \
  *listed = k_force_rb<EV, B, EV ? E : MINB, PF, KB, SH, P2, LPA>;
  switch (variant) {
    case 1: FMD_FORCE_VARIANT(4, 8, true, 2, 0, false, 1) break;
    case 2: FMD_FORCE_VARIANT(4, 8, true, 1, 1, false, 1) break;
    case 3: FMD_FORCE_VARIANT(4, 8, true, 2, 1, false, 1) break;
    case 4: FMD_FORCE_VARIANT(4, 8, true, 1, 1, true, 1) break;
    case 5: FMD_FORCE_VARIANT(4, 8, true, 2, 1, true, 1) break;
    case 6: FMD_FORCE_VARIANT(4, 7, true, 1, 1, true, 1) break;
    case 7: FMD_FORCE_VARIANT(4, 9, true, 1, 1, true, 1) break;
    case 8: FMD_FORCE_VARIANT(4, 6, true, 1, 1, false, 1) break;
    case 9: FMD_FORCE_VARIANT(4, 8, true, 1, 1, true, 2) break;
    case 10: FMD_FORCE_VARIANT(4, 8, true, 1, 1, true, 4) break;
    case 11: FMD_FORCE_VARIANT(4, 8, 3, 1, 1, true, 1) break;
    case 12: FMD_FORCE_VARIANT(4, 8, 4, 1, 1, true, 1) break;
    case 13: FMD_FORCE_VARIANT(4, 8, 2, 1, 1, true, 1) break;
    case 14: FMD_FORCE_VARIANT(4, 9, 2, 1, 1, true, 1) break;
    default: FMD_FORCE_VARIANT(4, 8, true, 1, 0, false, 1) break;
  }
#undef FMD_FORCE_VARIANT
}

// The force kernels use 4 KB of shared memory per block: ask for the
// smallest shared-memory carve-out, leaving the rest of the SM's unified
// L1 / shared array to cache the neighbor-position gathers.
template <typename K>
void prefer_l1(K kernel, int pct = kForceCarveoutPct) {
  FMD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
}

// The ring variants hold 4-8 KB of list rows per block besides the 2 KB of
// tables: carve-outs that keep 8 (9) of their blocks resident.
inline int force_carveout_pct(int variant) {
  return variant == 11 || variant == 12 ? 40 : variant == 13 || variant == 14 ? 28 : kForceCarveoutPct;
}

void launch_force(const Dev& d, int nchunks, bool ev, int variant, cudaStream_t st, bool skip_rebuilt) {
  void (*per_chunk)(Dev, int) = nullptr;
  void (*listed)(Dev) = nullptr;
  if (ev) force_kernels<true>(variant, &per_chunk, &listed);
  else force_kernels<false>(variant, &per_chunk, &listed);
  static bool set[2][kForceVariants] = {};
  const int v = variant >= 0 && variant < kForceVariants ? variant : 0;
  bool& done = set[ev ? 1 : 0][v];
  if (!done) {
    prefer_l1(per_chunk, force_carveout_pct(variant));
    prefer_l1(listed);
    done = true;
  }
  per_chunk<<<nchunks, kChunk, 0, st>>>(d, skip_rebuilt ? 1 : 0);
}

void launch_force_rebuilt(const Dev& d, bool ev, int variant, cudaStream_t st) {
  static int grid[2][kForceVariants] = {};
  void (*per_chunk)(Dev, int) = nullptr;
  void (*listed)(Dev) = nullptr;
  if (ev) force_kernels<true>(variant, &per_chunk, &listed);
  else force_kernels<false>(variant, &per_chunk, &listed);
  const int v = variant >= 0 && variant < kForceVariants ? variant : 0;
  int& g = grid[ev ? 1 : 0][v];
  if (!g) g = resident_grid(listed, kChunk);
  launch_hi(listed, g, kChunk, st, d);
}

void launch_forces_only(const Dev& d, int nchunks, int variant, bool has_table, cudaStream_t st) {
  launch_force(d, nchunks, false, variant, st, false);
  launch_force(d, nchunks, true, variant, st, false);
  if (has_table) {
    launch_table(d, nchunks, false, 0, st);
    launch_table(d, nchunks, true, 0, st);
  }
}
void launch_reduce_only(const Dev& d, int nchunks, int nreps, cudaStream_t st, int mode) {
  k_post<<<nchunks, kChunk, 0, st>>>(d, mode);
  k_post_commit<<<nreps, kPostCommitThreads, 0, st>>>(d, mode);
}

void launch_prepare(const Dev& d, int nreps, cudaStream_t st) { k_prepare<<<nreps, 32, 0, st>>>(d); }

}  // namespace mixed
}  // namespace fmd
