/*
 * fastmd_b200 — C ABI for the bead-spring MD per-step path on NVIDIA B200.
 *
 * The reference fastMD has two boundaries around this path, and this header
 * replaces both:
 *
 *  1. The process boundary `fastMD <run.conf>` (src/main.cu:24-36): run.conf
 *     keys (src/io/config.cpp:32-127), LAMMPS data input
 *     (src/io/lammps_data.cpp:18-229), thermo rows (src/analysis/thermo.cu:80,192)
 *     and rg rows (src/analysis/rg.cu:95,127-129).  fmd_sim_create() takes the
 *     same run.conf text and data file; fmd_thermo()/fmd_rg() return the values
 *     behind the same columns; fmd_format_thermo_row()/fmd_format_rg_row()
 *     produce the reference's text rows.
 *
 *  2. The in-process launchers that take raw device pointers and a stream
 *     (force/lj.cuh:4-12, force/fene.cuh:11-19, force/angle.cuh:9-15,
 *     neighbor/verlet_list.cuh:28-30, core/morton.cuh:17-18).  The fmd_launch_*
 *     entry points below accept the reference's own buffer layouts (float4 with
 *     the type id bit-cast into .w, int2 bonds, int4 angles, transposed Verlet
 *     list) so a caller of those launchers can switch one call at a time.
 *
 * Conventions (all functions):
 *  - Every function returns fmd_status; nothing calls exit().  On failure
 *    fmd_last_error() gives a message (thread-local).
 *  - Host buffers are caller-owned.  Device memory behind a handle is owned by
 *    the handle.  fmd_launch_* calls touch only caller-provided device memory
 *    plus the scratch the call names.
 *  - A handle is used by one host thread at a time; a server owns its thread.
 *  - Atom arrays in and out of fmd_sim/fmd_batch are in data-file order
 *    (the order atoms were given), regardless of the device storage order.
 */
#ifndef FASTMD_B200_H
#define FASTMD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FMD_API __attribute__((visibility("default")))
#else
#define FMD_API
#endif

typedef int32_t fmd_status;
enum {
  FMD_OK = 0,
  FMD_ERR_ARG = 1,       /* bad argument or handle */
  FMD_ERR_CONFIG = 2,    /* run.conf problem (reference: std::runtime_error, config.cpp:195-210) */
  FMD_ERR_IO = 3,        /* file or data-file problem (reference: lammps_data.cpp:21-49) */
  FMD_ERR_CUDA = 4,      /* CUDA runtime error (reference: CUDA_CHECK -> exit, types.cuh:7-15) */
  FMD_ERR_OVERFLOW = 5,  /* neighbor-list or cell capacity exceeded (reference truncates, verlet_list.cu:215) */
  FMD_ERR_TIMEOUT = 6,   /* a bounded device-side wait expired */
  FMD_ERR_FAULT = 7,     /* replica fault: non-finite state or FENE bond past R0 (reference clamps, fene.cu:33) */
  FMD_ERR_CAPACITY = 8,  /* batch slots or device-memory budget exhausted */
  FMD_ERR_NO_DEVICE = 9, /* no usable CUDA device */
  FMD_ERR_STATE = 10     /* call not valid in the current state */
};

/* Numerical form of a simulation. */
enum {
  FMD_FORM_PLAIN_FP64 = 0, /* mirrors the reference kernels and step loop in FP64, one system at a time */
  FMD_FORM_MIXED = 1       /* FP32 forces on cell-relative positions, FP64 reductions and thermostat
                              scalars; batched, device-side rebuilds, CUDA-graph step loop */
};

/* Ensembles (run.conf nvt_langevin / nvt_nh / npt_nh; config.cpp:76-97). */
enum { FMD_LANGEVIN = 0, FMD_NVT_NH = 1, FMD_NPT_NH = 2 };

/* Seeded Kremer-Grest melt: random-walk chains, then an optional capped-force
 * Langevin push-off.  All draws come from the library's Philox stream. */
typedef struct fmd_melt_spec {
  int32_t nchains;
  int32_t chain_length;
  double density;        /* beads per sigma^3; L = cbrt(N / density) */
  uint64_t seed;
  int32_t type_block;    /* > 0: types alternate 0,1 in blocks of this many beads along each chain */
  double bond_length;    /* random-walk step (0 -> 0.97) */
  double min_dist;       /* reject non-bonded beads closer than this (0 -> 0.8) */
  int32_t pushoff_steps; /* capped-force Langevin steps run on the device at creation (0 -> none) */
  double pushoff_fcap;   /* cap on each atom's non-bonded (LJ) force during push-off (0 -> 50) */
  double pushoff_dt;     /* push-off time step (0 -> 0.005) */
} fmd_melt_spec;

/* An in-memory system (what a LAMMPS data file carries). */
typedef struct fmd_system_desc {
  int32_t natoms;
  int32_t ntypes;        /* number of atom types (masses length) */
  double box_L;          /* cubic box edge; positions wrapped into [0, L) or unwrapped with images */
  const double* xyz;     /* [3N] */
  const double* vel;     /* [3N] or NULL (zero) */
  const int32_t* image;  /* [3N] or NULL (zero) */
  const int32_t* type;   /* [N] 0-based */
  const int32_t* mol;    /* [N] molecule ids or NULL (all 1) */
  const double* mass;    /* [ntypes] or NULL (all 1) */
  int32_t nbonds;
  const int32_t* bonds;  /* [2*nbonds] 0-based atom indices */
  const int32_t* bond_type;  /* [nbonds] 0-based */
  int32_t nangles;
  const int32_t* angles;     /* [3*nangles] i, j (vertex), k */
  const int32_t* angle_type; /* [nangles] */
} fmd_system_desc;

/* Values behind one thermo row (analysis/thermo.cu:140-195), in FP64.
 * stress[] is in the reference's emission order xx, xy, xz, yy, yz, zz (the
 * reference's header labels them Pxx Pyy Pzz Pxy Pxz Pyz). */
typedef struct fmd_thermo_row {
  int64_t step;
  double ke;        /* kinetic energy per atom */
  double pe;        /* potential energy per atom */
  double temp;      /* 2/3 KE per atom (no COM correction, thermo.cu:178) */
  double stress[6];
  double box_L;
  double conserved; /* extended energy per atom (thermostat / barostat terms included) */
} fmd_thermo_row;

typedef struct fmd_sim fmd_sim;
typedef struct fmd_batch fmd_batch;
typedef struct fmd_server fmd_server;

/* ---------------------------------------------------------------- library */
FMD_API const char* fmd_version(void);
FMD_API int32_t fmd_last_error(char* buf, size_t len);
FMD_API fmd_status fmd_device_count(int32_t* n);

/* ------------------------------------------------------- host-only helpers */
/* Generate a melt on the host (no push-off; no GPU needed).  First call with
 * out arrays NULL to get counts[0..2] = natoms, nbonds, nangles and *box_L. */
FMD_API fmd_status fmd_generate_melt(const fmd_melt_spec* spec, int32_t* counts, double* box_L,
                                     double* xyz, int32_t* image, int32_t* type, int32_t* mol,
                                     int32_t* bonds, int32_t* angles);
/* Parse run.conf text the way src/io/config.cpp:10-213 does.
 * iout: natoms, ntypes, nsteps, ensemble, chain_length, thermo_on, thermo_freq,
 *       rg_on, rg_freq, n_bond_types, n_angle_types
 * fout: rc, skin, dt, T_start, T_stop, Tdamp, P_start, P_stop, Pdamp
 * lj[ntypes*ntypes*2], bond[4*n_bond_types], angle[2*n_angle_types] (theta0 in radians). */
FMD_API fmd_status fmd_parse_run_conf(const char* text, int32_t* iout, double* fout, double* lj,
                                      int32_t lj_cap, double* bond, int32_t bond_cap, double* angle,
                                      int32_t angle_cap, uint64_t* seed);
/* Output and run-control keys of a run.conf (src/io/config.cpp:32-127; acted
 * on by src/main.cu:632-691, 738-783): what the `fastmd <run.conf>` program
 * writes and when.  restart_freq: -1 no restart files (the key absent), 0 the
 * final file only, > 0 also every restart_freq steps.  Strings are
 * NUL-terminated and truncated to their buffers. */
typedef struct fmd_output_spec {
  int64_t nsteps;
  int32_t ensemble;
  int32_t thermo_on, thermo_freq;
  int32_t rg_on, rg_freq;
  int32_t stress_on, stress_freq;
  int32_t dump_freq;
  int32_t restart_freq;
  char thermo_file[256];
  char rg_file[256];
  char stress_file[256];
  char restart_file[256];
  char data_file[256];
  char forces_dump_file[256];
} fmd_output_spec;
FMD_API fmd_status fmd_run_conf_outputs(const char* text, fmd_output_spec* out);
/* Restart file names of the reference (io/lammps_data.cpp:255-267): base
 * "restart.data" -> "restart_<step>.data" (step >= 0) or "restart_final.data"
 * (step < 0); without an extension the suffix is appended. */
FMD_API fmd_status fmd_restart_filename(const char* base, int64_t step, char* buf, size_t len);
/* Read one keyword section of a LAMMPS pair_style table file, as the
 * run.conf key 'table ti tj file keyword' does (io/table_parser.cpp:7-87):
 * grid = rmin, rmax, dr, inv_dr (single precision, as the reference derives
 * them); data = r, force, energy per point (cap points at most).  The force
 * column is applied as F/r, as force/table.cu:92-96 applies it. */
FMD_API fmd_status fmd_read_pair_table(const char* path, const char* keyword, float* grid, int32_t* npoints,
                                       float* data, int32_t cap);
/* Type pair -> table index of a run.conf ([ntypes*ntypes], -1: no table);
 * *ntables = distinct tables. */
FMD_API fmd_status fmd_run_conf_tables(const char* text, int32_t* table_of, int32_t cap, int32_t* ntables);
/* Read a LAMMPS data file (src/io/lammps_data.cpp:18-229).  First call with
 * xyz == NULL to get counts[0..3] = natoms, nbonds, nangles, ntypes. */
FMD_API fmd_status fmd_read_lammps_data(const char* path, int32_t* counts, double* box_L, double* xyz,
                                        int32_t* image, int32_t* type, int32_t* mol, double* vel,
                                        int32_t* bonds, int32_t* bond_type, int32_t* angles,
                                        int32_t* angle_type, double* masses);
/* Write a system as a LAMMPS data file in the layout of the reference's
 * restart writer (src/io/lammps_data.cpp:269-385): header with the step,
 * Masses, "Atoms # full" with image flags, Velocities, Bonds, Angles.  Values
 * carry 17 significant digits (the reference writes %.6f); the zhi line
 * carries the box edge (the reference's writer omits it, :335). */
FMD_API fmd_status fmd_write_lammps_data(const char* path, const fmd_system_desc* desc, int64_t step);
/* Reference text rows: "%d  %.4f ..." (thermo.cu:192) and "%d  %.4f" (rg.cu:127). */
FMD_API fmd_status fmd_format_thermo_row(const fmd_thermo_row* row, char* buf, size_t len);
FMD_API fmd_status fmd_format_rg_row(int64_t step, double rg, char* buf, size_t len);

/* ---------------------------------------------------------- one simulation */
/* Exactly one of data_path / desc / gen supplies the atoms.  data_path NULL and
 * desc NULL and gen NULL: use run.conf's lammps_data_file key. */
FMD_API fmd_status fmd_sim_create(const char* run_conf_text, const char* data_path,
                                  const fmd_system_desc* desc, const fmd_melt_spec* gen,
                                  int32_t form, fmd_sim** out);
FMD_API fmd_status fmd_sim_destroy(fmd_sim* sim);
FMD_API fmd_status fmd_sim_info(const fmd_sim* sim, int32_t* natoms, int32_t* nbonds,
                                int32_t* nangles, int64_t* step, double* box_L);
/* Advance nsteps (main.cu:403-736 semantics). */
FMD_API fmd_status fmd_step(fmd_sim* sim, int64_t nsteps);
/* Forces at the current positions: f[3N], pe[N] (per-atom share, as force.w),
 * virial[6] (xx,xy,xz,yy,yz,zz).  Any of the outputs may be NULL. */
FMD_API fmd_status fmd_compute_forces(fmd_sim* sim, double* f, double* pe, double* virial);
/* Wrapped positions in [0, L), velocities, image flags, in data-file order. */
FMD_API fmd_status fmd_get_state(fmd_sim* sim, double* xyz, double* vel, int32_t* image);
FMD_API fmd_status fmd_set_state(fmd_sim* sim, const double* xyz, const double* vel, const int32_t* image);
FMD_API fmd_status fmd_thermo(fmd_sim* sim, fmd_thermo_row* row);
/* Restart file of the current state (write_lammps_data, io/lammps_data.cpp:269;
 * main.cu:681-691, 738-745 call it every restart_freq steps and at the end),
 * plus a sidecar "<path>.state" with what the data file lacks: the step
 * counter (the Langevin noise is keyed on it), the Nose-Hoover chain and
 * barostat state, box edge and reference volume, and the list settings
 * (text, 17 significant digits).  Creating a simulation or a batch replica
 * from a data file that has a sidecar resumes from it.  A restart is a
 * checkpoint: the simulation continues from the state as written and
 * re-loaded (list rebuilt, forces re-evaluated), which is exactly what a
 * resumed run starts from, so run N + M equals run N, restart, run M: bit
 * for bit in the mixed form, to FP64 round-off in the plain form (whose
 * bonded forces are scattered with atomics, as the reference's are), in
 * every ensemble (the stress autocorrelator is not carried over).  The
 * reference writes only the data file. */
FMD_API fmd_status fmd_write_restart(fmd_sim* sim, const char* path);
/* Binary trajectory (the reference's dump format, io/dump.cu:12-56, file
 * "traj.bin" of run.conf dump_freq): header {int32 0x4D444247, int32 natoms,
 * int32 ntypes}, then per frame {int64 step, int32 natoms, float box_L,
 * float xyz[3 natoms]}, positions in atom-id order wrapped in the box of the
 * last pre-force update.  A frame of a batch replica is packed on the device
 * and copied into one of two pinned buffers; a background thread writes it,
 * so the call returns once the copy is queued. */
typedef struct fmd_traj fmd_traj;
FMD_API fmd_status fmd_traj_open(const char* path, int32_t natoms, int32_t ntypes, fmd_traj** out);
FMD_API fmd_status fmd_traj_write_sim(fmd_traj* t, fmd_sim* sim);
FMD_API fmd_status fmd_traj_write_batch(fmd_traj* t, fmd_batch* b, int32_t slot);
/* Writes the queued frames, closes the file and frees the handle. */
FMD_API fmd_status fmd_traj_close(fmd_traj* t);
/* Stress autocorrelation of a mixed-form simulation (see fmd_batch_stress_acf). */
FMD_API fmd_status fmd_stress_acf(fmd_sim* sim, int64_t* lag_steps, double* values, int64_t* counts, int32_t cap,
                                  int32_t* nrows);
FMD_API fmd_status fmd_write_stress_acf(fmd_sim* sim, const char* path);
FMD_API fmd_status fmd_rg(fmd_sim* sim, double* rg);
/* Current Verlet pair set (unordered pairs i < j within rc + skin at the last
 * rebuild, 1-2 bonded pairs excluded), in data-file indices. */
FMD_API fmd_status fmd_pairs(fmd_sim* sim, int32_t* i, int32_t* j, int64_t cap, int64_t* n);
/* Counters: rebuilds, device status word, neighbor-list capacity per atom. */
FMD_API fmd_status fmd_sim_counters(const fmd_sim* sim, int64_t* rebuilds, int32_t* status_word,
                                    int32_t* max_neighbors);

/* ------------------------------------------------------ batched replicas */
typedef struct fmd_batch_opts {
  int32_t device;          /* CUDA device ordinal */
  int32_t max_replicas;    /* slot count */
  int64_t max_atoms;       /* total atom capacity (padded); 0 -> sized from budget */
  double hbm_budget_gb;    /* device-memory budget for the batch (0 -> 150) */
  int32_t graph_steps;     /* steps captured per CUDA graph launch (0 -> 50; < 0: no graph) */
} fmd_batch_opts;

typedef struct fmd_replica_info {
  int32_t slot;
  int32_t natoms;
  int64_t step;
  int64_t nsteps;          /* run.conf nsteps (target) */
  int32_t status_word;     /* 0 healthy; bits: 1 overflow, 2 non-finite, 4 FENE overstretch, 8 cell capacity */
  int32_t active;
  double box_L;
  int64_t rebuilds;
} fmd_replica_info;

FMD_API fmd_status fmd_batch_create(const fmd_batch_opts* opts, fmd_batch** out);
FMD_API fmd_status fmd_batch_destroy(fmd_batch* b);
/* Admit a replica (run.conf text plus one atom source); returns its slot.
 * FMD_ERR_CAPACITY when no slot or memory is free. */
FMD_API fmd_status fmd_batch_add_replica(fmd_batch* b, const char* run_conf_text, const char* data_path,
                                         const fmd_system_desc* desc, const fmd_melt_spec* gen,
                                         int32_t* slot);
/* Bytes of device memory a replica would take (admission control). */
FMD_API fmd_status fmd_batch_estimate_bytes(const char* run_conf_text, int32_t natoms, double box_L,
                                            int64_t* bytes);
/* Advance every active replica by up to nsteps (a replica stops at its own
 * run.conf nsteps). */
FMD_API fmd_status fmd_batch_run(fmd_batch* b, int64_t nsteps);
FMD_API fmd_status fmd_batch_retire(fmd_batch* b, int32_t slot);
FMD_API fmd_status fmd_batch_replica_info(fmd_batch* b, int32_t slot, fmd_replica_info* info);
FMD_API fmd_status fmd_batch_get_state(fmd_batch* b, int32_t slot, double* xyz, double* vel, int32_t* image);
FMD_API fmd_status fmd_batch_thermo(fmd_batch* b, int32_t slot, fmd_thermo_row* row);
/* Restart data file and state sidecar of a replica (see fmd_write_restart);
 * fmd_batch_add_replica with that data file resumes from it.  Exact resume
 * also needs the same kernel variants (fmd_batch_set_variants). */
FMD_API fmd_status fmd_batch_write_restart(fmd_batch* b, int32_t slot, const char* path);
FMD_API fmd_status fmd_batch_rg(fmd_batch* b, int32_t slot, double* rg);
FMD_API fmd_status fmd_batch_compute_forces(fmd_batch* b, int32_t slot, double* f, double* pe, double* virial);
/* The geometry fmd_batch_compute_forces' forces belong to: positions (3N,
 * atom-id order) wrapped in the box of the last pre-force update, and that
 * box edge.  It is the current box except under NPT, whose post-force
 * barostat half step moves box_L before the next pre-force rescales the
 * positions (fmd_batch_get_state reports them re-wrapped into box_L). */
FMD_API fmd_status fmd_batch_get_force_frame(fmd_batch* b, int32_t slot, double* xyz, double* box_L);
/* Stress autocorrelation of a replica with run.conf 'stress <on> <freq>
 * <file>' (analysis/correlator.cu:33-92, output main.cu:758-783): the
 * pressure tensor of every stress step (columns xx, xy, xz, yy, yz, zz, as
 * in the thermo row) feeds a 16-level x 16-point multiple-tau correlator.
 * Rows in the reference file's order: lag in steps, 6 averaged products
 * (values[6 * row + c]) and the number of products.  *nrows = rows available
 * (up to 256); at most cap are copied. */
FMD_API fmd_status fmd_batch_stress_acf(fmd_batch* b, int32_t slot, int64_t* lag_steps, double* values,
                                        int64_t* counts, int32_t cap, int32_t* nrows);
/* The same rows as the reference's stress file ("# lag_steps  C_xx ... count"). */
FMD_API fmd_status fmd_batch_write_stress_acf(fmd_batch* b, int32_t slot, const char* path);
FMD_API fmd_status fmd_batch_pairs(fmd_batch* b, int32_t slot, int32_t* i, int32_t* j, int64_t cap, int64_t* n);
/* Totals: active replicas, atoms, device bytes in use. */
FMD_API fmd_status fmd_batch_totals(fmd_batch* b, int32_t* active, int64_t* atoms, int64_t* bytes);

/* Measurement hooks (device time on the batch's own stream).
 * fmd_batch_mark records CUDA event `which` (0 or 1) on the batch stream;
 * fmd_batch_elapsed_ms gives event1 - event0 after synchronizing.
 * fmd_batch_time_force re-evaluates the force kernel `iters` times on the
 * current state (idempotent) and returns its mean device time per launch.
 * fmd_batch_list_stats: total neighbor-list entries and the largest per-atom
 * count over active replicas.
 * fmd_batch_kernels_per_step: kernel launches one step issues at most.
 * fmd_batch_launch_counts: launches executed so far per kernel, counted on
 * the device (a graph step skips the rebuild kernels and a force variant no
 * replica needs): counts[0..12] = pre-force, bin, scan, scatter, cell sort,
 * permute, bonded tables, neighbor list, force, force with energies,
 * post-force, rebuild planning, per-replica commits; n = entries to fill. */
FMD_API fmd_status fmd_batch_mark(fmd_batch* b, int32_t which);
FMD_API fmd_status fmd_batch_elapsed_ms(fmd_batch* b, double* ms);
FMD_API fmd_status fmd_batch_time_force(fmd_batch* b, int32_t iters, double* ms_per_launch);
FMD_API fmd_status fmd_batch_list_stats(fmd_batch* b, int64_t* entries, int32_t* max_per_atom);
FMD_API fmd_status fmd_batch_kernels_per_step(fmd_batch* b, int32_t* n);
FMD_API fmd_status fmd_batch_launch_counts(fmd_batch* b, int64_t* counts, int32_t n);
/* Pruned pair list of a replica: the pairs of the rc + skin Verlet list
 * within rc + delta, re-filtered whenever a displacement since the last
 * filter exceeds delta / 2 (under NPT, (s (rc + delta) - rc) / 2 with s the
 * contraction since the filter), are what the force kernels walk (fewer
 * entries than the full list; a rebuild then waits for the displacement
 * since the rebuild, bounded by the filters' displacements, to reach
 * skin / 2).  On by default with delta = 0.12 in the mixed form when the
 * skin is wider; delta <= 0 turns it off.  A refinement of the reference's
 * single list (neighbor/verlet_list.cu), same forces up to summation order. */
FMD_API fmd_status fmd_batch_set_list_prune(fmd_batch* b, int32_t slot, double delta);
/* List buffer of a replica: the Verlet list holds the pairs within rc + skin
 * and is rebuilt after a displacement of skin / 2 (neighbor/verlet_list.cu,
 * neighbor/skin_trigger.cuh with the run.conf `skin`, its default).  Setting
 * it rebuilds the list at once; FMD_ERR_ARG when the list capacity sized at
 * fmd_batch_add cannot hold it.  fmd_batch_autotune widens it to the cell
 * edge for replicas with a pruned list (their forces walk the pruned list,
 * so a wider buffer only makes rebuilds rarer).  The forces do not depend on
 * it beyond summation order. */
FMD_API fmd_status fmd_batch_set_list_buffer(fmd_batch* b, int32_t slot, double skin);
FMD_API fmd_status fmd_batch_get_list_buffer(fmd_batch* b, int32_t slot, double* skin);
/* Autotuner: time each force-kernel variant (blocks per SM, batches per
 * compensated add, shift lookup, packed pair arithmetic, lanes per atom,
 * list words loaded ahead in registers or staged in a shared-memory ring)
 * `iters` times on the current state and each neighbor-list variant on a
 * full rebuild (ballot form with 8 or 6 blocks per SM, row form), keep the
 * fastest for all following steps.  chosen = force variant index;
 * ms_per_variant (cap entries, may be NULL) = device ms per launch of each
 * force variant (n_force of fmd_batch_get_variants), then ms per full
 * rebuild of each neighbor variant (n_nbr), then the chosen neighbor
 * variant.  It also lifts the forced rebuild
 * cadence of the active replicas (rebuilds then follow the skin/2
 * displacement trigger alone; fmd_batch_set_rebuild_cadence restores one)
 * and widens the list buffer of replicas with a pruned list to the cell
 * edge (fmd_batch_set_list_buffer restores the run.conf skin). */
FMD_API fmd_status fmd_batch_autotune(fmd_batch* b, int32_t iters, int32_t* chosen, double* ms_per_variant,
                                      int32_t cap);
/* Set the forced rebuild cadence of a replica (the reference rebuilds at
 * least every 20 steps, main.cu:401, the default here); the skin/2
 * displacement test still triggers rebuilds in between.  max_steps <= 0:
 * no forced cadence (skin trigger only, which is what fmd_batch_autotune
 * selects). */
FMD_API fmd_status fmd_batch_set_rebuild_cadence(fmd_batch* b, int32_t slot, int32_t max_steps);

/* Kernel variants (the autotuner's choices), for tests and for pinning a
 * choice: force_variant in [0, n_force), nbr_variant in [0, n_nbr); a value
 * < 0 keeps the current one.  Variants round the force sums differently in
 * the last bits (different batch and compensation groupings); each is
 * bit-reproducible.  No counterpart in the reference (one kernel each). */
FMD_API fmd_status fmd_batch_set_variants(fmd_batch* b, int32_t force_variant, int32_t nbr_variant);
FMD_API fmd_status fmd_batch_get_variants(fmd_batch* b, int32_t* force_variant, int32_t* nbr_variant,
                                          int32_t* n_force, int32_t* n_nbr);
/* Forces of the replica's last force evaluation as stored on the device (FP32
 * values, id order), without re-evaluating them: after a step these are the
 * forces the kernel flavour of that step produced at the positions of
 * fmd_batch_get_force_frame. */
FMD_API fmd_status fmd_batch_last_forces(fmd_batch* b, int32_t slot, double* f);

/* ------------------------------------------------------------- serving */
/* A request loop on its own host thread: submitted requests are admitted as
 * slots and the device-memory budget allow, advanced together in the batch,
 * retired when their run.conf nsteps is reached, and their slots back-filled. */
typedef struct fmd_server_opts {
  fmd_batch_opts batch;
  int32_t steps_per_round; /* steps between admission / retirement decisions (0 -> 200) */
} fmd_server_opts;

typedef struct fmd_request_result {
  int64_t request_id;
  fmd_status status;
  int32_t natoms;
  int64_t steps;
  double submit_time;      /* seconds, server clock */
  double start_time;
  double finish_time;
  fmd_thermo_row thermo;   /* final thermo values */
  double rg;               /* final mean chain Rg */
} fmd_request_result;

FMD_API fmd_status fmd_server_create(const fmd_server_opts* opts, fmd_server** out);
FMD_API fmd_status fmd_server_submit(fmd_server* s, const char* run_conf_text, const fmd_melt_spec* gen,
                                     int64_t* request_id);
/* Collect up to cap finished results; *n receives the count. */
FMD_API fmd_status fmd_server_poll(fmd_server* s, fmd_request_result* out, int32_t cap, int32_t* n);
/* queued, running, finished, atoms resident, atom-steps done. */
FMD_API fmd_status fmd_server_stats(fmd_server* s, int64_t* queued, int64_t* running, int64_t* finished,
                                    int64_t* atoms_resident, double* atom_steps);
/* Host seconds the batch thread spent admitting (upload, setup), stepping and
 * retiring (readouts), rounds run, and CUDA-graph captures so far. */
FMD_API fmd_status fmd_server_timing(fmd_server* s, double* admit_s, double* run_s, double* retire_s,
                                     int64_t* rounds, int64_t* graph_captures);
FMD_API fmd_status fmd_server_drain(fmd_server* s, double timeout_s);
FMD_API fmd_status fmd_server_destroy(fmd_server* s);

/* ---------------------------------------------------------- several GPUs */
/* The reference runs one system on one GPU; these spread independent
 * replicas over several (no data-path exchange between them).
 * fmd_partition_replicas: greedy longest-processing-time placement of n
 * replicas with the given costs (atom counts, or atoms x steps) on nparts
 * GPUs: replicas in decreasing cost (ties: lower index first), each to the
 * part with the least total cost so far (ties: lower part).  Deterministic,
 * so every process of a multi-process run computes the same placement.
 * part_of[n] receives each replica's part; part_cost[nparts] (may be NULL)
 * the total per part. */
FMD_API fmd_status fmd_partition_replicas(const int64_t* cost, int32_t n, int32_t nparts, int32_t* part_of,
                                          int64_t* part_cost);
/* A pool of request servers, one per listed device (each with its own host
 * thread, batch and CUDA-graph step loop; a device may be listed twice).  A
 * submitted request goes to the server with the least outstanding work
 * (atoms x run.conf nsteps of its requests not yet polled; ties: lowest
 * index); *server (may be NULL) receives that server's index in devices[].
 * Request ids are pool-wide; poll, stats and drain cover every server. */
typedef struct fmd_server_pool fmd_server_pool;
FMD_API fmd_status fmd_server_pool_create(const fmd_server_opts* opts, const int32_t* devices, int32_t ndevices,
                                          fmd_server_pool** out);
FMD_API fmd_status fmd_server_pool_submit(fmd_server_pool* p, const char* run_conf_text, const fmd_melt_spec* gen,
                                          int64_t* request_id, int32_t* server);
FMD_API fmd_status fmd_server_pool_poll(fmd_server_pool* p, fmd_request_result* out, int32_t cap, int32_t* n);
FMD_API fmd_status fmd_server_pool_stats(fmd_server_pool* p, int64_t* queued, int64_t* running, int64_t* finished,
                                         int64_t* atoms_resident, double* atom_steps);
FMD_API fmd_status fmd_server_pool_drain(fmd_server_pool* p, double timeout_s);
FMD_API fmd_status fmd_server_pool_destroy(fmd_server_pool* p);

/* ------------------------------------------- reference-layout launchers */
/* Cell list + full Verlet list, replacing VerletList::build
 * (neighbor/verlet_list.cuh:28-30, verlet_list.cu:337-376).  pos is float4
 * [natoms] with the type id bit-cast into .w; neighbors is the transposed
 * layout neighbors[k * natoms + i] with max_neighbors rows; exclusions are the
 * CSR of build_exclusions (lammps_data.cpp:231-253), or NULL.  Unlike the
 * reference, an overflow is reported (FMD_ERR_OVERFLOW after the stream is
 * synchronized when sync != 0) instead of truncated silently.
 * scratch: device memory of fmd_verlet_scratch_bytes() bytes. */
FMD_API fmd_status fmd_verlet_scratch_bytes(int32_t natoms, float rc_skin, float box_L, size_t* bytes);
FMD_API fmd_status fmd_launch_verlet_build(const void* pos, int32_t natoms, float box_L,
                                           const int32_t* exclusion_offsets, const int32_t* exclusion_list,
                                           float rc_skin, int32_t max_neighbors, int32_t* neighbors,
                                           int32_t* num_neighbors, void* scratch, size_t scratch_bytes,
                                           int32_t* overflow_flag, void* stream);
/* Allocation-free variant of fmd_launch_verlet_build; it has no counterpart in
 * the reference.  It is for callers that cannot allocate device memory: code
 * running inside another framework's memory pool, inside a stream-capture
 * region, or in a process that must keep its device footprint fixed after
 * start-up.  The caller still passes the positions, exclusions and output
 * buffers; the cell-list scratch lives in one static device array inside the
 * library (8 MiB, held by every GPU that loads the library until the process
 * exits).  Limits: natoms <= 131072 and at most 65536 cells (box_L / rc_skin
 * <= 40 per axis); larger inputs return FMD_ERR_CAPACITY, and a box_L or
 * rc_skin that is not finite and positive returns FMD_ERR_ARG, both before
 * anything is launched.  The first call on a device looks the array's address
 * up for that device (cudaGetSymbolAddress) and keeps it for the life of the
 * process, so make that first call before any stream capture; a
 * cudaDeviceReset of that device invalidates the kept address, and calls
 * after one are not supported.  Every call on a device
 * shares the one array and each call re-initialises what must start at zero,
 * so calls whose kernels overlap on the GPU (different streams, no ordering)
 * race; order them on one stream.  No cudaMalloc / cudaFree is called. */
FMD_API fmd_status fmd_launch_verlet_build_static(const void* pos, int32_t natoms, float box_L,
                                                  const int32_t* exclusion_offsets,
                                                  const int32_t* exclusion_list, float rc_skin,
                                                  int32_t max_neighbors, int32_t* neighbors,
                                                  int32_t* num_neighbors, int32_t* overflow_flag, void* stream);
/* LJ over the transposed list, replacing launch_lj_kernel (force/lj.cuh:4-12;
 * lj.cu:4-122): force[i] = (F, pe_i) overwritten, virial[6] accumulated. */
FMD_API fmd_status fmd_launch_lj(const void* pos, void* force, float* virial, const void* lj_params,
                                 const int32_t* neighbors, const int32_t* num_neighbors, int32_t natoms,
                                 int32_t ntypes, float rc2, float box_L, float inv_L, void* stream);
/* Tile list of 32-atom tiles, replacing TileList::build
 * (neighbor/tile_list.cuh:3-23, tile_list.cu:143-171): pairs of tiles (a, b),
 * ntiles = ceil(natoms / 32), whose axis-aligned boxes over the tiles'
 * positions lie within rc_skin (minimum image between the box centres,
 * tile_list.cu:63-99), as CSR: offsets[ntiles + 1] (device) and neighbors
 * (device, at most capacity) in increasing b for each a.  The reference
 * materialises ntiles^2 flags; this build uses O(ntiles) scratch
 * (fmd_tile_list_scratch_bytes).  npairs (host, may be NULL): the stream is
 * synchronised and the pair count returned; more pairs than capacity gives
 * FMD_ERR_OVERFLOW (the first capacity are written). */
FMD_API fmd_status fmd_tile_list_scratch_bytes(int32_t natoms, size_t* bytes);
FMD_API fmd_status fmd_launch_tile_list(const void* pos, int32_t natoms, float box_L, float rc_skin,
                                        int32_t* offsets, int32_t* neighbors, int32_t capacity, int32_t* npairs,
                                        void* scratch, size_t scratch_bytes, void* stream);
/* LJ over a tile list (offsets / neighbors as fmd_launch_tile_list writes
 * them, built at rc or beyond), a warp per 32-atom tile with each partner
 * tile staged in shared memory: a consumer of TileList's tile pairs
 * (neighbor/tile_list.cuh:3-23), which the reference defines but none of
 * its force kernels walks.  The same outputs and pair arithmetic as fmd_launch_lj
 * (force[i] = (F, pe_i) overwritten, virial[6] accumulated); the pairs are
 * every (i, j != i) within rc2 (minimum image) of the listed tile pairs,
 * less the exclusions: exclusion_offsets[natoms + 1] / exclusion_list in the
 * form fmd_launch_verlet_build_static takes (both NULL: none). */
FMD_API fmd_status fmd_launch_lj_tiles(const void* pos, void* force, float* virial, const void* lj_params,
                                       const int32_t* tile_offsets, const int32_t* tile_neighbors,
                                       const int32_t* exclusion_offsets, const int32_t* exclusion_list,
                                       int32_t natoms, int32_t ntypes, float rc2, float box_L, float inv_L,
                                       void* stream);
/* 30-bit Morton sort of pos and vel, replacing MortonSorter::sort_and_permute
 * (core/morton.cuh:17-18; morton.cu:65-85); the permutation is bit-exact with
 * a stable sort of (key, index).  perm (device, [padded natoms]) receives the
 * order.  scratch: fmd_morton_scratch_bytes() bytes. */
FMD_API fmd_status fmd_morton_scratch_bytes(int32_t natoms, size_t* bytes);
FMD_API fmd_status fmd_launch_morton_sort(void* pos, void* vel, int32_t natoms, float inv_L, int32_t* perm,
                                          void* scratch, size_t scratch_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FASTMD_B200_H */
