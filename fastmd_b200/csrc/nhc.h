// Nose-Hoover chain and MTK barostat scalar updates in double precision,
// shared by host and device code.  Operation order follows the reference:
//   chain half step: host nh_propagate_chain (integrate/nose_hoover.cu:356-447)
//                    and nh_propagate_chain_kernel (:86-178)
//   exponential:     6th-order Taylor nh_expf (:72-84), here in FP64
//   NPT barostat:    nh_npt_chain_baro_kernel (:185-305)
// All arithmetic uses the non-contracting helpers of counter_rng.h so host and
// device produce the same bits for the chain (the barostat's exp / cbrt /
// sinh come from the platform math library).
#pragma once
#include "counter_rng.h"

namespace fmd {

struct NHScalars {
  double xi[10];
  double vxi[10];
  double eps, veps;  // log strain and barostat momentum
  double carry;      // KE * scale^2 carried into the next pre-force half step
  double scale;      // latest thermostat velocity scale
  // barostat-derived values for the current step
  double L, inv_L, V;
  double bscale;     // exp(-(1 + 3/N_f) v_eps/W dt/2)
  double exp_vW;     // exp(v_eps/W dt)
  double vWdt;       // v_eps/W dt
  double fpos;       // dt exp(x) sinh(x)/x, x = vWdt/2
  double ke_raw;     // sum m v^2 of the last reduction
  double vir_tr;     // virial trace of the last reduction
  // Opt-in (run.conf nh_chain_carry 1): the chain's upper accelerations
  // carried from one half step to the next, as LAMMPS's fix nh keeps its
  // eta_dotdot; 0 follows the reference, which starts every half step from
  // zero (nose_hoover.cu:101, :251, :369).
  int32_t carry_dd;
  double dd[10];
};

FMD_HD double nh_exp6(double x) {
  const double x2 = FMD_DMUL(x, x), x3 = FMD_DMUL(x2, x), x4 = FMD_DMUL(x3, x), x5 = FMD_DMUL(x4, x),
               x6 = FMD_DMUL(x5, x);
  double s = FMD_DADD(1.0, x);
  s = FMD_DADD(s, FMD_DMUL(x2, 0.5));
  s = FMD_DADD(s, FMD_DMUL(x3, 1.0 / 6.0));
  s = FMD_DADD(s, FMD_DMUL(x4, 1.0 / 24.0));
  s = FMD_DADD(s, FMD_DMUL(x5, 1.0 / 120.0));
  s = FMD_DADD(s, FMD_DMUL(x6, 1.0 / 720.0));
  return s;
}

// One chain half step of length half_dt against total kinetic energy
// total_KE (= 0.5 sum m v^2); returns the velocity scale.  dd_keep: NULL
// for the reference's scheme, whose downward sweep drives the upper chain
// elements with zero accelerations (the array is reset every half step);
// otherwise the accelerations of the previous half step's upward sweep are
// read from it and this half step's are stored back (LAMMPS's eta_dotdot).
// The reset makes the chain update irreversible to first order in dt: with
// Tdamp = 100 dt the extended energy of a 600-bead melt gains about 1.5 kT
// per tau in NVT; carried, it stays flat.
FMD_HD double nhc_half_step(double* xi, double* vxi, int M, double Q1, double Qr, double kT, int natoms,
                            double total_KE, double half_dt, double* dd_keep = nullptr) {
  const double Nf = FMD_DMUL(3.0, (double)natoms);
  const double dt2 = half_dt, dt4 = FMD_DMUL(half_dt, 0.5), dt8 = FMD_DMUL(half_dt, 0.25);
  double dd[10];
  for (int k = 0; k < 10; ++k) dd[k] = (dd_keep && k > 0) ? dd_keep[k] : 0.0;
  double T = FMD_DDIV(FMD_DMUL(2.0, total_KE), Nf);
  if (Q1 > 0.0) dd[0] = FMD_DDIV(FMD_DSUB(FMD_DMUL(Nf, T), FMD_DMUL(Nf, kT)), Q1);
  const double ncfac = 1.0;
  for (int ich = M - 1; ich > 0; --ich) {
    const double ef = (ich + 1 < M) ? nh_exp6(FMD_DMUL(FMD_DMUL(-ncfac, dt8), vxi[ich + 1])) : 1.0;
    vxi[ich] = FMD_DMUL(vxi[ich], ef);
    vxi[ich] = FMD_DADD(vxi[ich], FMD_DMUL(FMD_DMUL(dd[ich], ncfac), dt4));
    vxi[ich] = FMD_DMUL(vxi[ich], ef);
  }
  const double ef0 = (M > 1) ? nh_exp6(FMD_DMUL(FMD_DMUL(-ncfac, dt8), vxi[1])) : 1.0;
  vxi[0] = FMD_DMUL(vxi[0], ef0);
  vxi[0] = FMD_DADD(vxi[0], FMD_DMUL(FMD_DMUL(dd[0], ncfac), dt4));
  vxi[0] = FMD_DMUL(vxi[0], ef0);
  const double fe = nh_exp6(FMD_DMUL(FMD_DMUL(-ncfac, dt2), vxi[0]));
  T = FMD_DMUL(T, FMD_DMUL(fe, fe));
  if (Q1 > 0.0) dd[0] = FMD_DDIV(FMD_DSUB(FMD_DMUL(Nf, T), FMD_DMUL(Nf, kT)), Q1);
  for (int ich = 0; ich < M; ++ich) xi[ich] = FMD_DADD(xi[ich], FMD_DMUL(FMD_DMUL(ncfac, dt2), vxi[ich]));
  vxi[0] = FMD_DMUL(vxi[0], ef0);
  vxi[0] = FMD_DADD(vxi[0], FMD_DMUL(FMD_DMUL(dd[0], ncfac), dt4));
  vxi[0] = FMD_DMUL(vxi[0], ef0);
  for (int ich = 1; ich < M; ++ich) {
    const double ef = (ich + 1 < M) ? nh_exp6(FMD_DMUL(FMD_DMUL(-ncfac, dt8), vxi[ich + 1])) : 1.0;
    vxi[ich] = FMD_DMUL(vxi[ich], ef);
    const double Qp = (ich == 1) ? Q1 : Qr;
    dd[ich] = FMD_DDIV(FMD_DSUB(FMD_DMUL(FMD_DMUL(Qp, vxi[ich - 1]), vxi[ich - 1]), kT), Qr);
    vxi[ich] = FMD_DADD(vxi[ich], FMD_DMUL(FMD_DMUL(dd[ich], ncfac), dt4));
    vxi[ich] = FMD_DMUL(vxi[ich], ef);
  }
  if (dd_keep)
    for (int k = 1; k < 10; ++k) dd_keep[k] = dd[k];
  return fe;
}

// NPT chain + barostat scalar update (nose_hoover.cu:185-305).  pre_force:
// barostat frozen, thermostat driven by the carried KE; otherwise a
// three-stage Suzuki-Yoshida update of (eps, v_eps) from P_inst, then the
// chain, and a new carry.  total_KE_raw is sum m v^2 (post-force only).
template <typename ExpF, typename CbrtF, typename SinhF>
FMD_HD void npt_chain_baro(NHScalars& s, bool pre_force, double total_KE_raw, double vir_tr, int M,
                           double Q1, double Qr, double W, double half_dt, double dt, double V0, int natoms,
                           double kT, double Pt, ExpF ex, CbrtF cb, SinhF sh) {
  const double Nf = 3.0 * (double)natoms;
  const double Nf_inv = 1.0 / Nf;
  double total_KE = pre_force ? s.carry : total_KE_raw * 0.5;
  double V = V0 * ex(3.0 * s.eps);
  if (!pre_force) {
    const double Pinst = (2.0 * total_KE + vir_tr) / (3.0 * V);
    const double c = cb(2.0);
    const double w3[3] = {1.0 / (2.0 - c), -c / (2.0 - c), 1.0 / (2.0 - c)};
    for (int sy = 0; sy < 3; ++sy) {
      const double w = w3[sy] * dt;
      double dv = 3.0 * V * (Pinst - Pt) * w;
      const double vh = s.veps + 0.5 * dv;
      s.eps += vh * w / W;
      dv = 3.0 * V0 * ex(3.0 * s.eps) * (Pinst - Pt) * w;
      s.veps += dv;
    }
    V = V0 * ex(3.0 * s.eps);
  }
  s.V = V;
  s.L = cb(V);
  s.inv_L = 1.0 / s.L;
  const double vW = s.veps / W;
  s.bscale = ex(-(1.0 + 3.0 * Nf_inv) * vW * half_dt);
  double KE = total_KE * s.bscale * s.bscale;
  s.exp_vW = ex(vW * dt);
  s.vWdt = vW * dt;
  const double hx = 0.5 * s.vWdt;
  const double sinhc = (hx < 1e-6 && hx > -1e-6) ? 1.0 + hx * hx / 6.0 : sh(hx) / hx;
  s.fpos = dt * ex(hx) * sinhc;
  s.scale = nhc_half_step(s.xi, s.vxi, M, Q1, Qr, kT, natoms, KE, half_dt, s.carry_dd ? s.dd : nullptr);
  if (!pre_force) s.carry = KE * s.scale * s.scale;
}

}  // namespace fmd
