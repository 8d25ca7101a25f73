/* FP64 CPU oracle for the bead-spring MD per-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and its --impl reference arm) use it, as the checker and as
 * the timed CPU baseline.
 *
 * It restates, in double precision, the algorithm of the reference fastMD
 * sources (paths relative to the fastMD project):
 *   core/pbc.cuh:4-28, core/morton.cu:4-28, reference/cpu_reference.hpp:7-53
 *   neighbor/verlet_list.cu:3-13, 58-104, 108-335, 337-376
 *   force/lj.cu:21-65, force/fene.cu:18-73, force/angle.cu:17-80
 *   integrate/langevin.cu:15-21, 34-130
 *   integrate/nose_hoover.cu:72-84, 86-305, 309-346, 356-447, 540-774, 780-898
 *   analysis/thermo.cu:88-195, analysis/rg.cu:3-69, main.cu:403-736
 * Each function in oracle.cpp cites the lines it follows.
 */
#ifndef FMD_ORACLE_H
#define FMD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system {
  int32_t natoms;
  int32_t ntypes;
  const int32_t* type;      /* [N] 0-based type ids */
  const int32_t* mol;       /* [N] molecule ids (may be NULL) */
  const double* mass;       /* [ntypes] */
  const double* lj;         /* [ntypes*ntypes*2] (eps, sig), row-major (ti, tj) */
  int32_t nbonds;
  const int32_t* bonds;     /* [2*nbonds] atom indices */
  const int32_t* bond_type; /* [nbonds] */
  int32_t nbond_types;
  const double* fene;       /* [nbond_types*4] k, R0, eps, sig */
  int32_t nangles;
  const int32_t* angles;    /* [3*nangles] i, j (vertex), k */
  const int32_t* angle_type;/* [nangles] */
  int32_t nangle_types;
  const double* angle_p;    /* [nangle_types*2] k_theta, theta0 (radians) */
  double rc;
  double skin;
  int32_t lj_clamp;         /* 1: clamp F/r to [-1000, 1000] as force/lj.cu:48 */
  int32_t fene_clamp;       /* 1: clamp r^2 to [1e-6, 0.9999 R0^2] as force/fene.cu:33 */
} orc_system;

enum { ORC_LANGEVIN = 0, ORC_NVT_NH = 1, ORC_NPT_NH = 2 };

typedef struct orc_run {
  int32_t ensemble;
  double dt;
  double T_start, T_stop, Tdamp;
  double P_start, P_stop, Pdamp;
  int32_t chain_length;
  uint64_t seed;
  int64_t nsteps;           /* ramp denominator (run.conf nsteps) */
  int32_t max_steps_between_rebuilds; /* 20 in main.cu:401 */
  double force_cap;         /* > 0: cap |F_i| (push-off); 0: off */
  int32_t nthreads;         /* OpenMP threads (0: default) */
  int32_t chain_carry;      /* 1: chain accelerations kept between half steps (LAMMPS); 0: the reference */
} orc_run;

typedef struct orc_sim orc_sim;

/* RNG: independent restatement of the library's counter-RNG specification. */
void orc_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]);
void orc_normal3(uint64_t seed, uint32_t stream, uint64_t step, uint32_t id, double out[3]);

/* PBC and Morton (core/pbc.cuh, core/morton.cu, cpu_reference.hpp) */
double orc_min_image(double dr, double L, double inv_L);
double orc_wrap(double x, double L, double inv_L);
float orc_min_image_f32(float dr, float L, float inv_L);
uint32_t orc_morton_key_f32(float x, float y, float z, float inv_L);
void orc_morton_sort_f32(const float* xyz, int32_t n, float inv_L, int32_t* perm);

/* Pair sets: unordered pairs (i < j) within rcs, 1-2 bonded pairs excluded. */
int64_t orc_pairs_brute(const double* xyz, int32_t n, double L, double rcs,
                        const int32_t* bonds, int32_t nbonds,
                        int32_t* pi, int32_t* pj, int64_t cap);
int64_t orc_tile_list_aabb(const float* pos4, int32_t natoms, float L, float rc_skin, int32_t* offsets,
                           int32_t* neighbors, int64_t cap);
int64_t orc_pairs_brute_f32(const float* xyz, int32_t n, float L, float rcs,
                            const int32_t* bonds, int32_t nbonds,
                            int32_t* pi, int32_t* pj, int64_t cap);
/* Per-atom full Verlet lists in the reference's traversal order
 * (neighbor/verlet_list.cu:108-335).  nbr is [n * max_nbr] row-major; counts
 * hold the untruncated count.  Returns the cell count per dimension. */
int32_t orc_verlet_lists(const double* xyz, int32_t n, double L, double rcs,
                         const int32_t* bonds, int32_t nbonds,
                         int32_t max_nbr, int32_t* nbr, int32_t* counts);

/* Forces: f [3N], pe [N] (per-atom share), vir [6] (xx,xy,xz,yy,yz,zz). */
int32_t orc_forces(const orc_system* sys, const double* xyz, double L,
                   double* f, double* pe, double* vir);
/* Individual terms, for closed-form checks. */
void orc_lj(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir);
void orc_fene(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir);
void orc_angle(const orc_system* sys, const double* xyz, double L, double* f, double* pe, double* vir);

/* Nose-Hoover chain half step (host nh_propagate_chain, nose_hoover.cu:356-447),
 * with the 6th-order Taylor exponential of nose_hoover.cu:72-84. */
void orc_nhc_half(double* xi, double* v_xi, int32_t M, double Q1, double Q_rest,
                  double kT, int32_t natoms, double total_KE, double half_dt,
                  double* scale_out);

/* Thermo row (analysis/thermo.cu:140-195): out[0..8] = KE/atom, PE/atom, T,
 * stress xx, xy, xz, yy, yz, zz (the reference's emission order). */
void orc_thermo(const double* vel, const int32_t* type, const double* mass,
                const double* pe, const double* vir, int32_t n, double L, double* out);
/* Mean chain Rg over molecules (analysis/rg.cu:3-69); chains are the groups
 * of equal mol id, in increasing mol id order. */
double orc_rg(const double* xyz, const int32_t* image, const int32_t* mol, int32_t n, double L);

/* Whole-step simulation mirroring main.cu:403-736. */
orc_sim* orc_sim_create(const orc_system* sys, const orc_run* run, double L,
                        const double* xyz, const double* vel, const int32_t* image);
int32_t orc_sim_step(orc_sim* s, int64_t nsteps);
void orc_sim_get(const orc_sim* s, double* xyz, double* vel, int32_t* image,
                 double* f, double* pe, double* vir);
/* scal[0..]: L, step, rebuilds, xi[0..9], v_xi[0..9], eps, v_eps, carry, nh_scale */
void orc_sim_scalars(const orc_sim* s, double* scal);
void orc_sim_thermo(const orc_sim* s, double* out9);
double orc_sim_rg(const orc_sim* s);
/* Extended energy: KE + PE + chain + barostat (+ P V for NPT), per atom. */
double orc_sim_conserved(const orc_sim* s);
double orc_sim_conserved_mtk(const orc_sim* s);
void orc_sim_destroy(orc_sim* s);

#ifdef __cplusplus
}
#endif
#endif
