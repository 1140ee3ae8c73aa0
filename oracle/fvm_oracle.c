/*
 * Plain-C oracle for fvmhd3d's per-timestep fluid hot path.
 * TEST INFRASTRUCTURE ONLY (see fvm_oracle.h).
 *
 * This file restates, in the reference's own operation order, the one-rank
 * step of the MPI tree:
 *   get_active_ptcl / Scheduler     MPI/iterate.cpp:12-56, MPI/Scheduler.h:33-154
 *   get_active_faces                MPI/iterate.cpp:58-93
 *   slope_limiter                   MPI/compute_reconstruction.cpp:201-602
 *   compute_update (+compute_flux,  MPI/compute_update.cpp:22-499, 973-1095,
 *     riemann_solver HLLD)            1097-1341
 *   compute_pvel                    MPI/compute_pvel.cpp:5-52
 *   compute_timesteps/adjust        MPI/compute_timestep.cpp:6-207
 *   collect_results /               MPI/distribute_work.cpp:537-797
 *     distribute_fluid_update_data
 *   compute_update0                 MPI/compute_update.cpp:695-970
 *   compute_reconstruction          MPI/compute_reconstruction.cpp:24-199
 *   collect_reconstruction          MPI/distribute_work.cpp:799-864
 * Expressions keep the reference's evaluation order so that, compiled with
 * the reference's floating-point flags, results agree bit for bit.
 */
#define _GNU_SOURCE
#include "fvm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define NF 10
enum { MASS = 0, MOMX, MOMY, MOMZ, ENER, WBX, WBY, WBZ, MPSI, MENTR };
enum { DENS = 0, VELX, VELY, VELZ, ETHM, BX, BY, BZ, PSI, ENTR };
enum { NO_BOUNDARY = 0, REFLECTING = 1, OUTFLOW = 2, DIOD = 3 };
enum { RUNGMAX = 32 };

#define HUGEV ((double)3.40282347e+38F)

static inline double sqr(double x) { return x * x; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline int imax(int a, int b) { return (a < b) ? b : a; }

struct fvo_ctx {
  fvo_params p;
  int ncell, nface;
  int *s1, *s2;
  double *fn, *fc, *cvol, *cc;
  long long *off;
  int *ids;
  /* scheduler (MPI/Scheduler.h:4-30) */
  double dt_tick;
  unsigned long long tsysU, tprevU;
  long long iteration;  /* system::iteration (MPI/iterate.cpp:117) */
  int min_rung, max_rung;
  double t_global;
  /* state */
  double *pos, *vel, *tlast, *tend, *volume;
  int *rung, *bnd;
  double *U, *dU, *Wrec;
  double *opos, *ovel;  /* orig_pos, orig_vel (correct(), MPI/set_problem.cpp:89-101) */
  float *divb;          /* divBi (MPI/distribute_work.cpp:681) */
  /* per-step work */
  unsigned char *active, *lngb, *hasngb;
  int *alist, nactive;
  int *flist, nflist;
};

/* ---- scheduler ---------------------------------------------------------- */

static int exp_of(double dt) { /* MPI/Scheduler.h:33-38 */
  uint64_t u;
  memcpy(&u, &dt, 8);
  return (int)((u >> 52) & 0xfff);
}
static double get_dt(const fvo_ctx *c, int rung) { /* MPI/Scheduler.h:101-104 */
  unsigned long long dtU = 1ULL << (RUNGMAX - 1 - rung);
  return c->dt_tick * (double)dtU;
}
static int get_rung(const fvo_ctx *c, double dt) { /* MPI/Scheduler.h:87-92 */
  int r = exp_of(c->p.dtmax) - exp_of(dt);
  return imax(r, c->min_rung);
}

/* ---- EOS hooks (ideal gas MPI/set_problem.cpp:123-137; disk
 *      MPI/problems/mri_disk3d.cpp:368-389) ----------------------------- */

static double pressure(const fvo_ctx *c, const double *W) {
  if (c->p.eos == 0) return c->p.gamma > 1.0 ? (c->p.gamma - 1.0) * W[ETHM] : W[ETHM];
  return W[ETHM];
}
static double entropy_from_ethm(const fvo_ctx *c, const double *W) {
  if (c->p.eos == 0) return (c->p.gamma - 1.0) * W[ETHM] / pow(W[DENS], c->p.gamma);
  return 1.0;
}
static double ethm_from_entropy(const fvo_ctx *c, const double *W) {
  if (c->p.eos == 0) return W[ENTR] * pow(W[DENS], c->p.gamma) / (c->p.gamma - 1.0);
  return -1.0;
}
static double ethm_update(const fvo_ctx *c, const double *W, int i) {
  if (c->p.eos == 0) return W[ETHM];
  const double *x = c->pos + 3 * (size_t)i;
  const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  return (c->p.iso_GM / r) * sqr(c->p.iso_cfac) * W[DENS];
}
static double extra_timestep(const fvo_ctx *c, int i) {
  if (c->p.eos == 0) return HUGEV;
  if (c->bnd[i] != NO_BOUNDARY) return HUGEV;
  const double *x = c->pos + 3 * (size_t)i, *v = c->vel + 3 * (size_t)i;
  const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  return c->p.courant * r / (1.0 / HUGEV + sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
}

/* ---- prim <-> cons (MPI/Fluid.h:55-129) --------------------------------- */

static void to_primitive(const double *U, double V, double *W) {
  const double iM = 1.0 / U[MASS];
  const double iV = 1.0 / V;
  W[DENS] = U[MASS] * iV;
  W[VELX] = U[MOMX] * iM;
  W[VELY] = U[MOMY] * iM;
  W[VELZ] = U[MOMZ] * iM;
  W[BX] = U[WBX] * iV;
  W[BY] = U[WBY] * iV;
  W[BZ] = U[WBZ] * iV;
  W[PSI] = U[MPSI] * iM;
  W[ENTR] = U[MENTR] * iM;
  W[ETHM] = U[ENER] * iV - 0.5 * (sqr(W[BX]) + sqr(W[BY]) + sqr(W[BZ])) -
            0.5 * (sqr(W[VELX]) + sqr(W[VELY]) + sqr(W[VELZ])) * W[DENS];
}
static void to_conservative(const double *W, double V, double *U) {
  const double M = W[DENS] * V;
  U[MASS] = W[DENS] * V;
  U[MOMX] = W[VELX] * M;
  U[MOMY] = W[VELY] * M;
  U[MOMZ] = W[VELZ] * M;
  U[WBX] = W[BX] * V;
  U[WBY] = W[BY] * V;
  U[WBZ] = W[BZ] * V;
  U[MPSI] = W[PSI] * M;
  U[MENTR] = W[ENTR] * M;
  U[ENER] = W[ETHM] * V + 0.5 * (sqr(W[BX]) + sqr(W[BY]) + sqr(W[BZ])) * V +
            0.5 * (sqr(W[VELX]) + sqr(W[VELY]) + sqr(W[VELZ])) * M;
}

/* ---- HLLD Riemann solver at face speed w (MPI/compute_update.cpp:1109-1341) */

static void riemann_hlld(double gamma, double *flux, double Bx, double w,
                         double dens_L, double pres_L, double ethm_L, double velx_L, double vely_L,
                         double velz_L, double By_L, double Bz_L, double dens_R, double pres_R,
                         double ethm_R, double velx_R, double vely_R, double velz_R, double By_R,
                         double Bz_R) {
  const double signBx = Bx == 0.0 ? 0.0 : (Bx > 0.0 ? +1.0 : -1.0);
  const double momx_L = dens_L * velx_L, momy_L = dens_L * vely_L, momz_L = dens_L * velz_L;
  const double momx_R = dens_R * velx_R, momy_R = dens_R * vely_R, momz_R = dens_R * velz_R;
  const double chalf = 0.5;
  const double B2_L = sqr(Bx) + sqr(By_L) + sqr(Bz_L);
  const double v2_L = sqr(velx_L) + sqr(vely_L) + sqr(velz_L);
  const double etot_L = ethm_L + chalf * (dens_L * v2_L + B2_L);
  const double B2_R = sqr(Bx) + sqr(By_R) + sqr(Bz_R);
  const double v2_R = sqr(velx_R) + sqr(vely_R) + sqr(velz_R);
  const double etot_R = ethm_R + chalf * (dens_R * v2_R + B2_R);
  const double gpl = gamma * pres_L, gpr = gamma * pres_R;
  const double gpbl = gpl + B2_L, gpbr = gpr + B2_R;
  const double cfl2 = gpbl / dens_L, cfr2 = gpbr / dens_R;
  const double cfmax = sqrt(dmax(cfl2, cfr2));
  const double S_L = dmin(velx_L, velx_R) - cfmax;
  const double S_R = dmax(velx_L, velx_R) + cfmax;
  const double pT_L = pres_L + chalf * B2_L, pT_R = pres_R + chalf * B2_R;
  const double iSM = 1.0 / ((S_R - velx_R) * dens_R - (S_L - velx_L) * dens_L);
  const double S_M = iSM * ((S_R - velx_R) * momx_R - (S_L - velx_L) * momx_L - pT_R + pT_L);
  const double ipTs = 1.0 / ((S_R - velx_R) * dens_R - (S_L - velx_L) * dens_L);
  const double pT_s = ipTs * ((S_R - velx_R) * dens_R * pT_L - (S_L - velx_L) * dens_L * pT_R +
                              dens_L * dens_R * (S_R - velx_R) * (S_L - velx_L) * (velx_R - velx_L));
  const double velx_L_s = S_M, velx_L_ss = S_M, velx_R_s = S_M, velx_R_ss = S_M;
  const double B2x = Bx * Bx;
  const double iSLmSM = 1.0 / (S_L - S_M), iSRmSM = 1.0 / (S_R - S_M);
  const double dens_L_s = dens_L * (S_L - velx_L) * iSLmSM;
  const double dens_R_s = dens_R * (S_R - velx_R) * iSRmSM;
  const double divL = dens_L * (S_L - velx_L) * (S_L - S_M) - B2x;
  const double divR = dens_R * (S_R - velx_R) * (S_R - S_M) - B2x;
  const double idivL = (divL != 0.0) ? 1.0 / divL : 0.0;
  const double idivR = (divR != 0.0) ? 1.0 / divR : 0.0;
  const double vely_L_s = vely_L - Bx * By_L * (S_M - velx_L) * idivL;
  const double velz_L_s = velz_L - Bx * Bz_L * (S_M - velx_L) * idivL;
  const double By_L_s = By_L * (dens_L * sqr(S_L - velx_L) - B2x) * idivL;
  const double Bz_L_s = Bz_L * (dens_L * sqr(S_L - velx_L) - B2x) * idivL;
  const double vely_R_s = vely_R - Bx * By_R * (S_M - velx_R) * idivR;
  const double velz_R_s = velz_R - Bx * Bz_R * (S_M - velx_R) * idivR;
  const double By_R_s = By_R * (dens_R * sqr(S_R - velx_R) - B2x) * idivR;
  const double Bz_R_s = Bz_R * (dens_R * sqr(S_R - velx_R) - B2x) * idivR;
  const double vB_L = velx_L * Bx + vely_L * By_L + velz_L * Bz_L;
  const double vB_L_s = velx_L_s * Bx + vely_L_s * By_L_s + velz_L_s * Bz_L_s;
  const double etot_L_s = ((S_L - velx_L) * etot_L - pT_L * velx_L + pT_s * S_M + Bx * (vB_L - vB_L_s)) * iSLmSM;
  const double vB_R = velx_R * Bx + vely_R * By_R + velz_R * Bz_R;
  const double vB_R_s = velx_R_s * Bx + vely_R_s * By_R_s + velz_R_s * Bz_R_s;
  const double etot_R_s = ((S_R - velx_R) * etot_R - pT_R * velx_R + pT_s * S_M + Bx * (vB_R - vB_R_s)) * iSRmSM;
  const double dens_L_ss = dens_L_s, dens_R_ss = dens_R_s;
  const double sDens_L_s = sqrt(dens_L_s), sDens_R_s = sqrt(dens_R_s);
  const double S_L_s = S_M - fabs(Bx / sDens_L_s);
  const double S_R_s = S_M + fabs(Bx / sDens_R_s);
  const double idsqroot = 1.0 / (sDens_L_s + sDens_R_s);
  const double vely_ss = idsqroot * (sDens_L_s * vely_L_s + sDens_R_s * vely_R_s + (By_R_s - By_L_s) * signBx);
  const double velz_ss = idsqroot * (sDens_L_s * velz_L_s + sDens_R_s * velz_R_s + (Bz_R_s - Bz_L_s) * signBx);
  const double By_ss = idsqroot * (sDens_L_s * By_R_s + sDens_R_s * By_L_s + sDens_L_s * sDens_R_s * (vely_R_s - vely_L_s) * signBx);
  const double Bz_ss = idsqroot * (sDens_L_s * Bz_R_s + sDens_R_s * Bz_L_s + sDens_L_s * sDens_R_s * (velz_R_s - velz_L_s) * signBx);
  const double vB_L_ss = velx_L_ss * Bx + vely_ss * By_ss + velz_ss * Bz_ss;
  const double etot_L_ss = etot_L_s - sDens_L_s * (vB_L_s - vB_L_ss) * signBx;
  const double vB_R_ss = velx_R_ss * Bx + vely_ss * By_ss + velz_ss * Bz_ss;
  const double etot_R_ss = etot_R_s + sDens_R_s * (vB_R_s - vB_R_ss) * signBx;
  const double Fdens_L = dens_L * velx_L;
  const double Fmomx_L = momx_L * velx_L + pT_L - B2x;
  const double Fmomy_L = momy_L * velx_L - Bx * By_L;
  const double Fmomz_L = momz_L * velx_L - Bx * Bz_L;
  const double Fetot_L = etot_L * velx_L + pT_L * velx_L - Bx * vB_L;
  const double Fdens_R = dens_R * velx_R;
  const double Fmomx_R = momx_R * velx_R + pT_R - B2x;
  const double Fmomy_R = momy_R * velx_R - Bx * By_R;
  const double Fmomz_R = momz_R * velx_R - Bx * Bz_R;
  const double Fetot_R = etot_R * velx_R + pT_R * velx_R - Bx * vB_R;
  const double momx_L_s = dens_L_s * velx_L_s, momy_L_s = dens_L_s * vely_L_s, momz_L_s = dens_L_s * velz_L_s;
  const double momx_L_ss = dens_L_ss * velx_L_ss, momy_L_ss = dens_L_ss * vely_ss, momz_L_ss = dens_L_ss * velz_ss;
  const double momx_R_s = dens_R_s * velx_R_s, momy_R_s = dens_R_s * vely_R_s, momz_R_s = dens_R_s * velz_R_s;
  const double momx_R_ss = dens_R_ss * velx_R_ss, momy_R_ss = dens_R_ss * vely_ss, momz_R_ss = dens_R_ss * velz_ss;
  const double Fby_L = By_L * velx_L - Bx * vely_L, Fbz_L = Bz_L * velx_L - Bx * velz_L;
  const double Fby_R = By_R * velx_R - Bx * vely_R, Fbz_R = Bz_R * velx_R - Bx * velz_R;
  const int w_lt_SL = w <= S_L, w_le_SLs = w <= S_L_s, w_le_SM = w <= S_M;
  const int w_le_SRs = w <= S_R_s, w_le_SR = w <= S_R;
  const double fdens = w_le_SM ? Fdens_L : Fdens_R;
  const double fetot = w_le_SM ? Fetot_L : Fetot_R;
  const double fmomx = w_le_SM ? Fmomx_L : Fmomx_R;
  const double fmomy = w_le_SM ? Fmomy_L : Fmomy_R;
  const double fmomz = w_le_SM ? Fmomz_L : Fmomz_R;
  const double fby = w_le_SM ? Fby_L : Fby_R;
  const double fbz = w_le_SM ? Fbz_L : Fbz_R;
  const double a = w_le_SLs ? 0.0 : (w_le_SM ? S_L_s - w : (w_le_SRs ? S_R_s - w : 0.0));
  const double b = w_lt_SL ? 0.0
                 : (w_le_SLs ? +S_L - w
                 : (w_le_SM ? -S_L_s + S_L
                 : (w_le_SRs ? -S_R_s + S_R : (w_le_SR ? +S_R - w : 0.0))));
  const double cc = w_lt_SL ? -w
                  : (w_le_SLs ? -S_L : (w_le_SM ? -S_L : (w_le_SRs ? -S_R : (w_le_SR ? -S_R : -w))));
  const double dens = w_le_SM ? dens_L : dens_R;
  const double dens_s = w_le_SM ? dens_L_s : dens_R_s;
  const double dens_ss = w_le_SM ? dens_L_ss : dens_R_ss;
  const double etot = w_le_SM ? etot_L : etot_R;
  const double etot_s = w_le_SM ? etot_L_s : etot_R_s;
  const double etot_ss = w_le_SM ? etot_L_ss : etot_R_ss;
  const double momx = w_le_SM ? momx_L : momx_R;
  const double momx_s = w_le_SM ? momx_L_s : momx_R_s;
  const double momx_ss = w_le_SM ? momx_L_ss : momx_R_ss;
  const double momy = w_le_SM ? momy_L : momy_R;
  const double momy_s = w_le_SM ? momy_L_s : momy_R_s;
  const double momy_ss = w_le_SM ? momy_L_ss : momy_R_ss;
  const double momz = w_le_SM ? momz_L : momz_R;
  const double momz_s = w_le_SM ? momz_L_s : momz_R_s;
  const double momz_ss = w_le_SM ? momz_L_ss : momz_R_ss;
  const double by = w_le_SM ? By_L : By_R;
  const double by_s = w_le_SM ? By_L_s : By_R_s;
  const double by_ss = w_le_SM ? By_ss : By_ss;
  const double bz = w_le_SM ? Bz_L : Bz_R;
  const double bz_s = w_le_SM ? Bz_L_s : Bz_R_s;
  const double bz_ss = w_le_SM ? Bz_ss : Bz_ss;
  flux[MASS] = fdens + a * dens_ss + b * dens_s + cc * dens;
  flux[ENER] = fetot + a * etot_ss + b * etot_s + cc * etot;
  flux[MOMX] = fmomx + a * momx_ss + b * momx_s + cc * momx;
  flux[MOMY] = fmomy + a * momy_ss + b * momy_s + cc * momy;
  flux[MOMZ] = fmomz + a * momz_ss + b * momz_s + cc * momz;
  flux[WBY] = fby + a * by_ss + b * by_s + cc * by;
  flux[WBZ] = fbz + a * bz_ss + b * bz_s + cc * bz;
  flux[WBX] = -w * Bx;
}

/* ---- rotated-frame face flux (MPI/compute_update.cpp:973-1095) ---------- */

static void compute_flux(const fvo_ctx *c, const double *wij, const double *Wi, const double *Wj,
                         int jbnd, const double *normal, double *psi_ij, double *Bn_ij,
                         double *flux) {
  const double gamma = c->p.gamma;
  const double ex = normal[0], ey = normal[1], ez = normal[2];
  const double ds = sqrt(ex * ex + ey * ey);
  const double ids = (ds != 0.0) ? 1.0 / ds : 0.0;
  const double cosph = (ids == 0.0) ? 1.0 : ex * ids;
  const double sinph = (ids == 0.0) ? 0.0 : ey * ids;
  const double costh = ez, sinth = ds;
  const double Axx = cosph * sinth, Axy = sinth * sinph, Axz = costh;
  const double Ayx = -sinph, Ayy = cosph, Ayz = 0.0;
  const double Azx = -costh * cosph, Azy = -costh * sinph, Azz = sinth;
  const double dens_L = Wi[DENS], ethm_L = Wi[ETHM];
  const double velx_L = Axx * Wi[VELX] + Axy * Wi[VELY] + Axz * Wi[VELZ];
  const double vely_L = Ayx * Wi[VELX] + Ayy * Wi[VELY] + Ayz * Wi[VELZ];
  const double velz_L = Azx * Wi[VELX] + Azy * Wi[VELY] + Azz * Wi[VELZ];
  const double Bx_L = Axx * Wi[BX] + Axy * Wi[BY] + Axz * Wi[BZ];
  const double By_L = Ayx * Wi[BX] + Ayy * Wi[BY] + Ayz * Wi[BZ];
  const double Bz_L = Azx * Wi[BX] + Azy * Wi[BY] + Azz * Wi[BZ];
  const double psiL = Wi[PSI], entrL = Wi[ENTR];
  const double dens_R = Wj[DENS], ethm_R = Wj[ETHM];
  double velx_R = Axx * Wj[VELX] + Axy * Wj[VELY] + Axz * Wj[VELZ];
  const double vely_R = Ayx * Wj[VELX] + Ayy * Wj[VELY] + Ayz * Wj[VELZ];
  const double velz_R = Azx * Wj[VELX] + Azy * Wj[VELY] + Azz * Wj[VELZ];
  const double Bx_R = Axx * Wj[BX] + Axy * Wj[BY] + Axz * Wj[BZ];
  const double By_R = Ayx * Wj[BX] + Ayy * Wj[BY] + Ayz * Wj[BZ];
  const double Bz_R = Azx * Wj[BX] + Azy * Wj[BY] + Azz * Wj[BZ];
  const double psiR = Wj[PSI], entrR = Wj[ENTR];
  const double pres_L = pressure(c, Wi), pres_R = pressure(c, Wj);
  const double wn_ij = Axx * wij[0] + Axy * wij[1] + Axz * wij[2];
  if (jbnd == REFLECTING) velx_R = -velx_R;
  else if (jbnd == DIOD) velx_R = dmax(velx_R - 1.2 * wn_ij, 0.0) + 1.2 * wn_ij;
  const double cfl2 = (gamma * pres_L + sqr(Bx_L) + sqr(By_L) + sqr(Bz_L)) / dens_L;
  const double cfr2 = (gamma * pres_R + sqr(Bx_R) + sqr(By_R) + sqr(Bz_R)) / dens_R;
  const double chL = sqrt(cfl2 + 0.0 * sqr(velx_L - wn_ij));
  const double chR = sqrt(cfr2 + 0.0 * sqr(velx_R - wn_ij));
  *Bn_ij = (Bx_L * chL + Bx_R * chR + (psiL - psiR)) / (chL + chR);
  *psi_ij = (psiL * chR + psiR * chL + chR * chL * (Bx_L - Bx_R)) / (chL + chR);
  double F[NF];
  riemann_hlld(gamma, F, *Bn_ij, wn_ij, dens_L, pres_L, ethm_L, velx_L, vely_L, velz_L, By_L, Bz_L,
               dens_R, pres_R, ethm_R, velx_R, vely_R, velz_R, By_R, Bz_R);
  const double iAxx = cosph * sinth, iAxy = -sinph, iAxz = -costh * cosph;
  const double iAyx = sinth * sinph, iAyy = cosph, iAyz = -costh * sinph;
  const double iAzx = costh, iAzy = 0.0, iAzz = sinth;
  flux[MASS] = F[MASS];
  flux[ENER] = F[ENER];
  flux[MOMX] = iAxx * F[MOMX] + iAxy * F[MOMY] + iAxz * F[MOMZ];
  flux[MOMY] = iAyx * F[MOMX] + iAyy * F[MOMY] + iAyz * F[MOMZ];
  flux[MOMZ] = iAzx * F[MOMX] + iAzy * F[MOMY] + iAzz * F[MOMZ];
  flux[WBX] = iAxx * F[WBX] + iAxy * F[WBY] + iAxz * F[WBZ];
  flux[WBY] = iAyx * F[WBX] + iAyy * F[WBY] + iAyz * F[WBZ];
  flux[WBZ] = iAzx * F[WBX] + iAzy * F[WBY] + iAzz * F[WBZ];
  flux[MPSI] = F[MASS] * (F[MASS] > 0.0 ? psiL : psiR);
  flux[MENTR] = F[MASS] * (F[MASS] > 0.0 ? entrL : entrR);
}

/* ---- limiter (MPI/compute_reconstruction.cpp:5-22) ---------------------- */

static double Phi(double x) {
  const double fac = 0.2, eps1 = 1.0e-16;
  return (x * x + 2.0 * x + fac * eps1) / (x * x + x + 2.0 + fac * eps1);
}
static double limiter(double dWi, double dWj_min, double dWj_max) {
  if (fabs(dWi) <= 1.0e-16 * dmax(fabs(dWj_max), fabs(dWj_min))) return 1.0;
  else if (dWi < 0.0) return Phi(dWj_min / dWi);
  else return Phi(dWj_max / dWi);
}

/* ---- helpers ------------------------------------------------------------ */

#define CELL3(a, i) ((a) + 3 * (size_t)(i))
#define WREC(c, i) ((c)->Wrec + 50 * (size_t)(i))
#define UU(c, i) ((c)->U + 10 * (size_t)(i))
#define DU(c, i) ((c)->dU + 14 * (size_t)(i))

static inline int ngb_of(const fvo_ctx *c, int f, int i) { return i == c->s1[f] ? c->s2[f] : c->s1[f]; }
static inline double face_area(const double *n) { return sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]); }

/* ---- API ----------------------------------------------------------------- */

fvo_ctx *fvo_create(const fvo_params *p) {
  fvo_ctx *c = (fvo_ctx *)calloc(1, sizeof(fvo_ctx));
  c->p = *p;
  c->dt_tick = p->dtmax / (double)(1ULL << (RUNGMAX - 1));
  c->tsysU = 0;
  c->min_rung = 0;
  c->max_rung = RUNGMAX - 1;
  return c;
}

static void free_state(fvo_ctx *c) {
  free(c->pos); free(c->vel); free(c->tlast); free(c->tend); free(c->volume);
  free(c->rung); free(c->bnd); free(c->U); free(c->dU); free(c->Wrec);
  free(c->active); free(c->lngb); free(c->hasngb); free(c->alist); free(c->flist);
  free(c->opos); free(c->ovel); free(c->divb);
}

void fvo_destroy(fvo_ctx *c) {
  if (!c) return;
  free(c->s1); free(c->s2); free(c->fn); free(c->fc); free(c->cvol); free(c->cc);
  free(c->off); free(c->ids);
  free_state(c);
  free(c);
}

int fvo_set_mesh(fvo_ctx *c, int ncell, int nface, const int *s1, const int *s2, const double *fn,
                 const double *fc, const double *cvol, const double *cc, const long long *off,
                 const int *ids) {
  c->ncell = ncell;
  c->nface = nface;
  c->s1 = (int *)malloc(sizeof(int) * nface);
  c->s2 = (int *)malloc(sizeof(int) * nface);
  c->fn = (double *)malloc(sizeof(double) * 3 * nface);
  c->fc = (double *)malloc(sizeof(double) * 3 * nface);
  c->cvol = (double *)malloc(sizeof(double) * ncell);
  c->cc = (double *)malloc(sizeof(double) * 3 * ncell);
  c->off = (long long *)malloc(sizeof(long long) * (ncell + 1));
  c->ids = (int *)malloc(sizeof(int) * off[ncell]);
  memcpy(c->s1, s1, sizeof(int) * nface);
  memcpy(c->s2, s2, sizeof(int) * nface);
  memcpy(c->fn, fn, sizeof(double) * 3 * nface);
  memcpy(c->fc, fc, sizeof(double) * 3 * nface);
  memcpy(c->cvol, cvol, sizeof(double) * ncell);
  memcpy(c->cc, cc, sizeof(double) * 3 * ncell);
  memcpy(c->off, off, sizeof(long long) * (ncell + 1));
  memcpy(c->ids, ids, sizeof(int) * off[ncell]);
  const size_t n = ncell;
  c->pos = (double *)calloc(3 * n, sizeof(double));
  c->vel = (double *)calloc(3 * n, sizeof(double));
  c->tlast = (double *)calloc(n, sizeof(double));
  c->tend = (double *)calloc(n, sizeof(double));
  c->volume = (double *)calloc(n, sizeof(double));
  c->rung = (int *)calloc(n, sizeof(int));
  c->bnd = (int *)calloc(n, sizeof(int));
  c->U = (double *)calloc(10 * n, sizeof(double));
  c->dU = (double *)calloc(14 * n, sizeof(double));
  c->Wrec = (double *)calloc(50 * n, sizeof(double));
  c->opos = (double *)calloc(3 * n, sizeof(double));
  c->ovel = (double *)calloc(3 * n, sizeof(double));
  c->divb = (float *)calloc(n, sizeof(float));
  c->active = (unsigned char *)calloc(n, 1);
  c->lngb = (unsigned char *)calloc(n, 1);
  c->hasngb = (unsigned char *)calloc(n, 1);
  c->alist = (int *)malloc(sizeof(int) * n);
  c->flist = (int *)malloc(sizeof(int) * (nface > 0 ? nface : 1));
  return 0;
}

/* compute_pvel (MPI/compute_pvel.cpp:5-52) for the cells in alist; with
 * static_mesh the compute_pvel1 hook that zeroes the velocity of every active
 * site and returns true (MPI/set_problem.cpp:61-72). */
static void compute_pvel(fvo_ctx *c) {
  if (c->p.static_mesh) {
    for (int a = 0; a < c->nactive; a++) memset(CELL3(c->vel, c->alist[a]), 0, 3 * sizeof(double));
    return;
  }
  for (int a = 0; a < c->nactive; a++) {
    const int i = c->alist[a];
    double W[NF];
    to_primitive(UU(c, i), c->volume[i], W);
    double *v = CELL3(c->vel, i);
    v[0] = W[VELX]; v[1] = W[VELY]; v[2] = W[VELZ];
    const double B2 = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
    const double pres = pressure(c, W);
    const double cs2 = (c->p.gamma * pres + B2) / W[DENS];
    const double vel2 = W[VELX] * W[VELX] + W[VELY] * W[VELY] + W[VELZ] * W[VELZ];
    const double vabs = sqrt(cs2 + vel2);
    const double *cc = CELL3(c->cc, i), *x = CELL3(c->pos, i);
    const double d3[3] = {cc[0] - x[0], cc[1] - x[1], cc[2] - x[2]};
    const double d = sqrt(d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2]);
    if (d == 0.0) continue;
    const double eta = 0.25f, ki = 1.0f, f1 = 0.9f, f2 = 1.1f;
    const double R = pow(c->cvol[i] * (3.0 / (4.0 * M_PI)), 1.0 / 3.0);
    const double fac = d / (eta * R);
    double f;
    if (fac < f1) f = 0.0;
    else if (fac < f2) f = (d - f1 * eta * R) / ((f2 - f1) * eta * R);
    else f = 1.0;
    const double tau = d / vabs;
    f *= ki / tau;
    v[0] += d3[0] * f; v[1] += d3[1] * f; v[2] += d3[2] * f;
    if (c->bnd[i] != NO_BOUNDARY) { v[0] = v[1] = v[2] = 0.0; }
  }
}

/* compute_timestep(i) (MPI/compute_timestep.cpp:6-51); i0 < 0 selects the
 * face-free form used by the shared-timestep initialisation */
static double compute_timestep(const fvo_ctx *c, int i0) {
  const int i = i0 < 0 ? -1 - i0 : i0;
  double W[NF];
  to_primitive(UU(c, i), c->volume[i], W);
  const double *pv = CELL3(c->vel, i);
  double csi = 0.0, vrel = 0.0;
  if (c->bnd[i] == NO_BOUNDARY) {
    const double Pi = pressure(c, W) * c->p.gamma;
    const double B2i = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
    csi = sqrt((Pi + B2i) / W[DENS]);
    const double s = (i0 < 0 ? 0.0 : 1.0);
    const double d[3] = {W[VELX] - pv[0] * s, W[VELY] - pv[1] * s, W[VELZ] - pv[2] * s};
    vrel = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  }
  const double V = c->volume[i];
  const double h = pow(V / (4.0 * M_PI / 3.0), 1.0 / 3.0);
  double dti = h / (csi + vrel + 1.0 / HUGEV);
  if (i0 >= 0) {
    const double fac = c->bnd[i] != NO_BOUNDARY ? 0.0 : 1.0;
    for (long long q = c->off[i]; q < c->off[i + 1]; q++) {
      const int j = ngb_of(c, c->ids[q], i);
      const double *vj = CELL3(c->vel, j);
      const double w3[3] = {(vj[0] + pv[0]) * 0.5, (vj[1] + pv[1]) * 0.5, (vj[2] + pv[2]) * 0.5};
      const double dw[3] = {vj[0] - pv[0], vj[1] - pv[1], vj[2] - pv[2]};
      const double r[3] = {W[VELX] - w3[0], W[VELY] - w3[1], W[VELZ] - w3[2]};
      const double rv = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const double dwa = sqrt(dw[0] * dw[0] + dw[1] * dw[1] + dw[2] * dw[2]);
      dti = dmin(dti, h / dmax(fac * (csi + rv), 1.0 / HUGEV + dwa));
    }
  }
  dti *= c->p.courant;
  return dti;
}

int fvo_init_problem(fvo_ctx *c, const double *W, const double *pos, const int *bnd, int rung_offset) {
  const int n = c->ncell;
  for (int i = 0; i < n; i++) {
    memcpy(CELL3(c->pos, i), pos + 3 * (size_t)i, 3 * sizeof(double));
    memset(CELL3(c->vel, i), 0, 3 * sizeof(double));
    c->tlast[i] = 0.0;
    c->tend[i] = 0.0;
    c->rung[i] = 0;
    c->bnd[i] = bnd ? bnd[i] : 0;
    c->volume[i] = c->cvol[i];
    double *r = WREC(c, i);
    memset(r, 0, 50 * sizeof(double));
    memcpy(r, W + 10 * (size_t)i, 10 * sizeof(double));
    to_conservative(W + 10 * (size_t)i, c->cvol[i], UU(c, i));
    memset(DU(c, i), 0, 14 * sizeof(double));
  }
  /* get_active_ptcl(true) + compute_pvel + compute_timesteps(true)
   * (MPI/problems/mri_disk3d.cpp:841-856; MPI/compute_timestep.cpp:57-75) */
  c->nactive = n;
  for (int i = 0; i < n; i++) c->alist[i] = i;
  compute_pvel(c);
  double dt_loc = HUGEV;
  for (int i = 0; i < n; i++) {
    const double dti = dmin(extra_timestep(c, i), compute_timestep(c, -1 - i));
    c->rung[i] = get_rung(c, dti);
    dt_loc = dmin(dt_loc, dti);
  }
  const int rung = get_rung(c, dt_loc);
  for (int i = 0; i < n; i++) {
    c->rung[i] = rung + rung_offset;
    c->tend[i] = 0.0 + get_dt(c, c->rung[i]);
    memcpy(CELL3(c->opos, i), CELL3(c->pos, i), 3 * sizeof(double));
    memcpy(CELL3(c->ovel, i), CELL3(c->vel, i), 3 * sizeof(double));
    c->divb[i] = 0.0f;
  }
  c->t_global = 0.0;
  return 0;
}

double fvo_time(const fvo_ctx *c) { return c->t_global; }

/* Scheduler::tsysU, the dt_global that pull_active_list returned
 * (MPI/Scheduler.h:138,153) and system::iteration. */
int fvo_clock(const fvo_ctx *c, unsigned long long *tsys, double *dt_global, long long *iteration) {
  if (tsys) *tsys = c->tsysU;
  if (dt_global) *dt_global = c->dt_tick * (double)(c->tsysU - c->tprevU);
  if (iteration) *iteration = c->iteration;
  return 0;
}

int fvo_get_motion(const fvo_ctx *c, double *opos, double *ovel, float *divb) {
  const size_t n = c->ncell;
  if (opos) memcpy(opos, c->opos, 3 * n * sizeof(double));
  if (ovel) memcpy(ovel, c->ovel, 3 * n * sizeof(double));
  if (divb) memcpy(divb, c->divb, n * sizeof(float));
  return 0;
}

int fvo_get_state(const fvo_ctx *c, double *pos, double *vel, double *tlast, double *tend, int *rung,
                  double *U, double *dU, double *wrec) {
  const size_t n = c->ncell;
  if (pos) memcpy(pos, c->pos, 3 * n * sizeof(double));
  if (vel) memcpy(vel, c->vel, 3 * n * sizeof(double));
  if (tlast) memcpy(tlast, c->tlast, n * sizeof(double));
  if (tend) memcpy(tend, c->tend, n * sizeof(double));
  if (rung) memcpy(rung, c->rung, n * sizeof(int));
  if (U) memcpy(U, c->U, 10 * n * sizeof(double));
  if (dU) memcpy(dU, c->dU, 14 * n * sizeof(double));
  if (wrec) memcpy(wrec, c->Wrec, 50 * n * sizeof(double));
  return 0;
}

int fvo_set_state(fvo_ctx *c, const double *vel, const double *tlast, const double *tend,
                  const int *rung, const double *U, const double *dU, const double *wrec,
                  unsigned long long tsys_ticks) {
  const size_t n = c->ncell;
  if (vel) memcpy(c->vel, vel, 3 * n * sizeof(double));
  if (tlast) memcpy(c->tlast, tlast, n * sizeof(double));
  if (tend) memcpy(c->tend, tend, n * sizeof(double));
  if (rung) memcpy(c->rung, rung, n * sizeof(int));
  if (U) memcpy(c->U, U, 10 * n * sizeof(double));
  if (dU) memcpy(c->dU, dU, 14 * n * sizeof(double));
  if (wrec) memcpy(c->Wrec, wrec, 50 * n * sizeof(double));
  c->tsysU = c->tprevU = tsys_ticks;
  c->t_global = c->dt_tick * (double)tsys_ticks;
  return 0;
}

static void copy_wrec_all(const fvo_ctx *c, const double *wtmp, double *out) {
  if (out) memcpy(out, wtmp, 50 * (size_t)c->ncell * sizeof(double));
}

/* One one-rank iterate_step on the fixed mesh (see file header). */
int fvo_step(fvo_ctx *c, int shared, fvo_snap *snap) {
  const int n = c->ncell;
  const double gamma = c->p.gamma;

  /* -- Scheduler::pull_active_list (MPI/Scheduler.h:108-154) -- */
  int max_rung = 0;
  for (int i = 0; i < n; i++) max_rung = imax(max_rung, c->rung[i]);
  c->max_rung = max_rung;
  const unsigned long long dtU = 1ULL << (RUNGMAX - 1 - max_rung);
  const unsigned long long tnextU = (c->tsysU / dtU + 1) * dtU;
  const unsigned long long flags = c->tsysU ^ tnextU;
  for (int b = 0; b < RUNGMAX; b++)
    if (flags & (1ULL << b)) c->min_rung = RUNGMAX - 1 - b;
  c->tprevU = c->tsysU;
  c->tsysU = tnextU;
  c->iteration++;
  c->t_global = c->dt_tick * (double)c->tsysU;
  const double t_global = c->t_global;

  /* -- active set, site flags (MPI/build_mesh_active.cpp:524-528) -- */
  c->nactive = 0;
  for (int i = 0; i < n; i++) {
    c->active[i] = (flags >> (RUNGMAX - 1 - c->rung[i])) & 1ULL;
    c->lngb[i] = c->hasngb[i] = 0;
  }
  for (int i = 0; i < n; i++) {
    if (!c->active[i]) continue;
    c->alist[c->nactive++] = i;
    for (long long q = c->off[i]; q < c->off[i + 1]; q++) {
      const int j = ngb_of(c, c->ids[q], i);
      if (!c->active[j]) { c->lngb[j] = 1; c->hasngb[i] = 1; }
    }
  }

  /* -- get_active_faces (MPI/iterate.cpp:58-93) -- */
  {
    unsigned char *seen = (unsigned char *)calloc(c->nface > 0 ? c->nface : 1, 1);
    c->nflist = 0;
    for (int a = 0; a < c->nactive; a++) {
      const int i = c->alist[a];
      if (c->bnd[i] != NO_BOUNDARY) continue;
      for (long long q = c->off[i]; q < c->off[i + 1]; q++) {
        const int f = c->ids[q];
        if (seen[f]) continue;
        seen[f] = 1;
        c->flist[c->nflist++] = f;
      }
    }
    free(seen);
  }
  if (snap && snap->nactive_faces) *snap->nactive_faces = c->nflist;
  if (snap && snap->active_faces) memcpy(snap->active_faces, c->flist, sizeof(int) * c->nflist);

  /* working copies of the import arrays: the reference mutates copies
   * (Wrec_import, ptcl_import, dU_import) and collects some of them back */
  double *wrec = (double *)malloc(50 * (size_t)n * sizeof(double));
  memcpy(wrec, c->Wrec, 50 * (size_t)n * sizeof(double));
  double *dUi = (double *)malloc(14 * (size_t)n * sizeof(double));
  memcpy(dUi, c->dU, 14 * (size_t)n * sizeof(double));
  double *Ui = (double *)malloc(10 * (size_t)n * sizeof(double));
  memcpy(Ui, c->U, 10 * (size_t)n * sizeof(double));
  int *rungi = (int *)malloc(sizeof(int) * n);
  memcpy(rungi, c->rung, sizeof(int) * n);
  double *tendi = (double *)malloc(sizeof(double) * n);
  memcpy(tendi, c->tend, sizeof(double) * n);
  double *voli = (double *)malloc(sizeof(double) * n);
  memcpy(voli, c->volume, sizeof(double) * n);
  double *veli = (double *)malloc(3 * sizeof(double) * n);
  memcpy(veli, c->vel, 3 * sizeof(double) * n);
  const double *tl = c->tlast;

  /* ======== slope_limiter (MPI/compute_reconstruction.cpp:201-602) ======== */
  {
    double *mm = (double *)malloc(20 * (size_t)n * sizeof(double)); /* min[10], max[10] */
    double *lim = (double *)malloc(10 * (size_t)n * sizeof(double));
    double *sdt = (double *)malloc(sizeof(double) * n);
    double *dtij = (double *)malloc(2 * sizeof(double) * (c->nflist > 0 ? c->nflist : 1));
    for (int i = 0; i < n; i++) {
      if (c->active[i] || c->lngb[i]) {
        sdt[i] = t_global - tl[i];
        for (int k = 0; k < NF; k++) { lim[10 * i + k] = 1.0; mm[20 * i + k] = mm[20 * i + 10 + k] = 0.0; }
      } else sdt[i] = -1.0;
    }
    for (int ff = 0; ff < c->nflist; ff++) {
      const int f = c->flist[ff];
      const int i = c->s1[f], j = c->s2[f];
      if (c->bnd[i] != NO_BOUNDARY || c->bnd[j] != NO_BOUNDARY) continue;
      const double dtI = sdt[i], dtJ = sdt[j];
      const double dth = 0.5 * dmin(dtI, dtJ);
      dtij[2 * ff] = dtI - dth;
      dtij[2 * ff + 1] = dtJ - dth;
      const double *wi = wrec + 50 * (size_t)i, *wj = wrec + 50 * (size_t)j;
      for (int k = 0; k < NF; k++) {
        const double diff = wj[k] - wi[k];
        mm[20 * i + k] = dmin(mm[20 * i + k], diff);
        mm[20 * i + 10 + k] = dmax(mm[20 * i + 10 + k], diff);
        mm[20 * j + k] = dmin(mm[20 * j + k], -diff);
        mm[20 * j + 10 + k] = dmax(mm[20 * j + 10 + k], -diff);
      }
    }
    for (int ff = 0; ff < c->nflist; ff++) {
      const int f = c->flist[ff];
      const int i = c->s1[f], j = c->s2[f];
      if (c->bnd[i] != NO_BOUNDARY || c->bnd[j] != NO_BOUNDARY) {
        for (int k = 0; k < NF; k++) lim[10 * i + k] = lim[10 * j + k] = 0;
        continue;
      }
      const double *x = CELL3(c->pos, i), *fc = c->fc + 3 * (size_t)f, *fn = c->fn + 3 * (size_t)f;
      const double dri[3] = {fc[0] - x[0], fc[1] - x[1], fc[2] - x[2]};
      const double area = face_area(fn);
      const double ia = 1.0 / area;
      const double nrm[3] = {fn[0] * ia, fn[1] * ia, fn[2] * ia};
      const double dsh = dri[0] * nrm[0] + dri[1] * nrm[1] + dri[2] * nrm[2];
      const double dsl = 2.0 * dsh;
      const double drj[3] = {dri[0] - nrm[0] * dsl, dri[1] - nrm[1] * dsl, dri[2] - nrm[2] * dsl};
      const double *ri = wrec + 50 * (size_t)i, *rj = wrec + 50 * (size_t)j;
      for (int k = 0; k < NF; k++) {
        const double dWit = ri[40 + k] * dtij[2 * ff];
        const double dWix = ri[10 + k] * dri[0] + ri[20 + k] * dri[1] + ri[30 + k] * dri[2];
        const double dWi = dWix + dWit;
        lim[10 * i + k] = dmin(lim[10 * i + k], limiter(dWi, mm[20 * i + k], mm[20 * i + 10 + k]));
        const double dWjt = rj[40 + k] * dtij[2 * ff + 1];
        const double dWjx = rj[10 + k] * drj[0] + rj[20 + k] * drj[1] + rj[30 + k] * drj[2];
        const double dWj = dWjx + dWjt;
        lim[10 * j + k] = dmin(lim[10 * j + k], limiter(dWj, mm[20 * j + k], mm[20 * j + 10 + k]));
      }
    }
    for (int i = 0; i < n; i++) {
      if (!(c->active[i] || c->lngb[i])) continue;
      double *r = wrec + 50 * (size_t)i;
      for (int k = 0; k < NF; k++) {
        const double tau = lim[10 * i + k];
        r[10 + k] *= tau; r[20 + k] *= tau; r[30 + k] *= tau; r[40 + k] *= tau;
      }
    }
    free(mm); free(lim); free(sdt); free(dtij);
  }
  if (snap) copy_wrec_all(c, wrec, snap->wrec_after_limiter);

  /* ======== compute_update (MPI/compute_update.cpp:22-499) ======== */
  int *failed = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int nfailed = 0;
  {
    double *dU0 = (double *)malloc(14 * (size_t)n * sizeof(double));
    memcpy(dU0, dUi, 14 * (size_t)n * sizeof(double));
    for (int i = 0; i < n; i++)
      if (c->active[i] || c->lngb[i]) memset(dUi + 14 * (size_t)i, 0, 14 * sizeof(double));
    for (int ff = 0; ff < c->nflist; ff++) {
      const int f = c->flist[ff];
      int i = c->s1[f], j = c->s2[f];
      const double *fn = c->fn + 3 * (size_t)f, *fc = c->fc + 3 * (size_t)f;
      const double area = face_area(fn);
      const double ia = 1.0 / area;
      double nrm[3] = {fn[0] * ia, fn[1] * ia, fn[2] * ia};
      const double *xi = CELL3(c->pos, i);
      double dri[3] = {fc[0] - xi[0], fc[1] - xi[1], fc[2] - xi[2]};
      if (c->bnd[i] != NO_BOUNDARY) {
        int t = i; i = j; j = t;
        for (int a = 0; a < 3; a++) { nrm[a] *= -1.0; dri[a] *= -1.0; }
      }
      const double *ri = wrec + 50 * (size_t)i, *rj = wrec + 50 * (size_t)j;
      const double dtI = t_global - tl[i], dtJ = t_global - tl[j];
      const double dt = dmin(dtI, dtJ);
      const double dti = dtI - 0.5 * dt, dtj = dtJ - 0.5 * dt;
      const double dsh = dri[0] * nrm[0] + dri[1] * nrm[1] + dri[2] * nrm[2];
      const double dsl = 2.0 * dsh;
      const double drj[3] = {dri[0] - nrm[0] * dsl, dri[1] - nrm[1] * dsl, dri[2] - nrm[2] * dsl};
      double Wi[NF], Wj[NF];
      if (c->bnd[j] != NO_BOUNDARY) {
        for (int k = 0; k < NF; k++) Wi[k] = Wj[k] = ri[k];
      } else {
        for (int k = 0; k < NF; k++) {
          Wi[k] = ri[k] + ((ri[10 + k] * dri[0] + ri[20 + k] * dri[1] + ri[30 + k] * dri[2]) + ri[40 + k] * dti);
          Wj[k] = rj[k] + ((rj[10 + k] * drj[0] + rj[20 + k] * drj[1] + rj[30 + k] * drj[2]) + rj[40 + k] * dtj);
        }
      }
      const double *vi = CELL3(c->vel, i), *vj = CELL3(c->vel, j);
      const double vij[3] = {vj[0] + vi[0], vj[1] + vi[1], vj[2] + vi[2]};
      const double dvij[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
      const double fij[3] = {dri[0] - nrm[0] * dsh, dri[1] - nrm[1] * dsh, dri[2] - nrm[2] * dsh};
      const double fdv = dvij[0] * fij[0] + dvij[1] * fij[1] + dvij[2] * fij[2];
      const double ids2 = -0.5 * fdv * ((dsh > 0.0) ? 1.0 / sqr(dsh) : 0.0);
      const double wij[3] = {vij[0] * 0.5 + dri[0] * ids2, vij[1] * 0.5 + dri[1] * ids2, vij[2] * 0.5 + dri[2] * ids2};
      double psi, Bn, flux[NF];
      compute_flux(c, wij, Wi, Wj, c->bnd[j], nrm, &psi, &Bn, flux);
      const double tarea = dt * area;
      const double dPsi[3] = {nrm[0] * (psi * tarea), nrm[1] * (psi * tarea), nrm[2] * (psi * tarea)};
      double *di = dUi + 14 * (size_t)i, *dj = dUi + 14 * (size_t)j;
      for (int k = 0; k < NF; k++) di[k] -= flux[k] * tarea;
      di[10] = di[10] + dPsi[0]; di[11] = di[11] + dPsi[1]; di[12] = di[12] + dPsi[2];
      di[13] += Bn * tarea;
      if (c->bnd[j] != NO_BOUNDARY) continue;
      for (int k = 0; k < NF; k++) dj[k] += flux[k] * tarea;
      dj[10] = dj[10] - dPsi[0]; dj[11] = dj[11] - dPsi[1]; dj[12] = dj[12] - dPsi[2];
      dj[13] -= Bn * tarea;
    }
    for (int a = 0; a < c->nactive; a++) {
      const int i = c->alist[a];
      if (c->bnd[i] != NO_BOUNDARY) { voli[i] = c->cvol[i]; continue; }
      double Uc[NF];
      const double *d0 = dU0 + 14 * (size_t)i;
      double *dn = dUi + 14 * (size_t)i;
      for (int k = 0; k < NF; k++) Uc[k] = Ui[10 * (size_t)i + k] + (d0[k] + dn[k]);
      const double divB = d0[13] + dn[13];
      const double dPsi[3] = {d0[10] + dn[10], d0[11] + dn[11], d0[12] + dn[12]};
      const double dt = t_global - tl[i];
      for (int k = 0; k < NF; k++) dn[k] = 0.0;
      dn[13] = dt > 0.0 ? divB / dt / c->cvol[i] : divB;
      dn[10] = dn[11] = dn[12] = 0.0;
      if (Uc[MASS] <= 0.0) { failed[nfailed++] = i; continue; }
      {
        const double *r = wrec + 50 * (size_t)i;
        const double dth = 0.5 * dt;
        double Wh[NF];
        for (int k = 0; k < NF; k++) Wh[k] = r[k] + r[40 + k] * dth;
        Uc[WBX] -= Wh[VELX] * divB;
        Uc[WBY] -= Wh[VELY] * divB;
        Uc[WBZ] -= Wh[VELZ] * divB;
        const double pres = pressure(c, Wh);
        const double B2 = Wh[BX] * Wh[BX] + Wh[BY] * Wh[BY] + Wh[BZ] * Wh[BZ];
        const double dcs2 = gamma * pres + B2;
        const double ch_sig = sqrt(dcs2 / Wh[DENS]);
        Uc[WBX] -= dPsi[0];
        Uc[WBY] -= dPsi[1];
        Uc[WBZ] -= dPsi[2];
        Uc[MPSI] -= dcs2 * divB;
        const double cr = 0.5;
        const double l_min = pow(c->cvol[i] / (4.0 * M_PI / 3.0), 1.0 / 3.0);
        Uc[MPSI] *= exp(-cr * ch_sig / l_min * dt);
      }
      voli[i] = c->cvol[i];
      double W1[NF];
      to_primitive(Uc, c->cvol[i], W1);
      W1[ETHM] = ethm_update(c, W1, i);
      if (W1[ETHM] <= 0.0) W1[ETHM] = ethm_from_entropy(c, W1);
      else W1[ENTR] = entropy_from_ethm(c, W1);
      to_conservative(W1, c->cvol[i], Ui + 10 * (size_t)i);
    }
    for (int q = 0; q < nfailed; q++) { /* MPI/compute_update.cpp:438-468 */
      const int i = failed[q];
      const double dt = t_global - tl[i];
      const double *r = wrec + 50 * (size_t)i;
      double W1[NF], Utmp[NF];
      for (int k = 0; k < NF; k++) W1[k] = r[k] + r[40 + k] * dt;
      to_conservative(W1, voli[i], Utmp);
      to_primitive(Utmp, c->cvol[i], W1);
      voli[i] = c->cvol[i];
      W1[ETHM] = ethm_update(c, W1, i);
      if (W1[ETHM] <= 0.0) W1[ETHM] = ethm_from_entropy(c, W1);
      else W1[ENTR] = entropy_from_ethm(c, W1);
      to_conservative(W1, c->cvol[i], Ui + 10 * (size_t)i);
    }
    free(dU0);
  }
  if (snap && snap->dU_after_update) memcpy(snap->dU_after_update, dUi, 14 * (size_t)n * sizeof(double));
  if (snap && snap->U_after_update) memcpy(snap->U_after_update, Ui, 10 * (size_t)n * sizeof(double));

  /* ======== compute_pvel ======== */
  {
    /* compute_pvel reads U_import and ptcl_import */
    double *Us = c->U, *vs = c->volume, *vls = c->vel;
    c->U = Ui; c->volume = voli; c->vel = veli;
    compute_pvel(c);
    c->U = Us; c->volume = vs; c->vel = vls;
  }
  if (snap && snap->vel_after_pvel) memcpy(snap->vel_after_pvel, veli, 3 * sizeof(double) * n);

  /* ======== compute_timesteps(false) + adjust_timesteps ======== */
  {
    double *dtl = (double *)malloc(sizeof(double) * n);
    const double dtfac = -1.0;
    for (int i = 0; i < n; i++) {
      dtl[i] = HUGEV;
      if (c->active[i] || c->lngb[i])
        dtl[i] = (tendi[i] - tl[i]) * (c->bnd[i] != NO_BOUNDARY ? dtfac : +1.0);
    }
    double dt_min = HUGEV;
    {
      double *Us = c->U, *vs = c->volume, *vls = c->vel;
      c->U = Ui; c->volume = voli; c->vel = veli;
      for (int a = 0; a < c->nactive; a++) {
        const int i = c->alist[a];
        dtl[i] = dmin(extra_timestep(c, i), compute_timestep(c, i));
        dt_min = dmin(dt_min, dtl[i]);
        if (c->bnd[i] != NO_BOUNDARY) dtl[i] = dtfac * dtl[i];
      }
      c->U = Us; c->volume = vs; c->vel = vls;
    }
    for (int a = 0; a < c->nactive; a++) {
      const int i = c->alist[a];
      if (dtl[i] >= 8.0 * dt_min) dtl[i] *= 0.5;
    }
    /* adjust_timesteps (MPI/compute_timestep.cpp:115-207) */
    unsigned char *hash = (unsigned char *)calloc(n > 0 ? n : 1, 1);
    for (int a = 0; a < c->nactive; a++) {
      const int i = c->alist[a];
      if (c->bnd[i] != NO_BOUNDARY) continue;
      for (long long q = c->off[i]; q < c->off[i + 1]; q++) {
        const int j = ngb_of(c, c->ids[q], i);
        if (dtl[j] < 0.0) continue;
        hash[j] = 1;
        dtl[i] = dmin(dtl[i], 2.0 * dtl[j]);
        dtl[j] = dmin(dtl[j], 2.0 * dtl[i]);
      }
    }
    unsigned char *wreset = (unsigned char *)calloc(n > 0 ? n : 1, 1);
    for (int i = 0; i < n; i++) {
      if (!(c->active[i] || c->lngb[i])) continue;
      if (c->active[i]) {
        rungi[i] = get_rung(c, fabs(dtl[i]));
      } else if (hash[i]) {
        const double tlast = tl[i], tend = tendi[i];
        if ((tend - tlast) > dtl[i]) {
          const int rr = imax(exp_of(c->p.dtmax) - exp_of(fabs(0.5 * dtl[i])), 0);
          const double dt = get_dt(c, rr);
          if (tlast + dt <= t_global) {
            rungi[i] = get_rung(c, dt);
            tendi[i] = t_global + get_dt(c, rungi[i]);
            rungi[i] = -1 - rungi[i];
          } else {
            rungi[i] = rr;
            tendi[i] = tlast + dt;
          }
        }
      }
    }
    if (snap && snap->rung_after_timestep) memcpy(snap->rung_after_timestep, rungi, sizeof(int) * n);
    if (snap && snap->dt_after_timestep) memcpy(snap->dt_after_timestep, dtl, sizeof(double) * n);

    if (shared) {
      int rmax = 0;
      for (int a = 0; a < c->nactive; a++) rmax = imax(rmax, rungi[c->alist[a]]);
      for (int a = 0; a < c->nactive; a++) rungi[c->alist[a]] = rmax;
    }

    /* ======== collect_results (MPI/distribute_work.cpp:657-722) ======== */
    for (int i = 0; i < n; i++) {
      if (!(c->active[i] || c->lngb[i])) continue;
      if (c->active[i]) {
        memcpy(UU(c, i), Ui + 10 * (size_t)i, 10 * sizeof(double));
        memset(DU(c, i), 0, 14 * sizeof(double));
        c->rung[i] = rungi[i];
        c->volume[i] = voli[i];
        memcpy(CELL3(c->vel, i), CELL3(veli, i), 3 * sizeof(double));
        c->tend[i] = tendi[i];
        c->divb[i] = (float)dUi[14 * (size_t)i + 13];
        /* correct(i), MPI/set_problem.cpp:89-101 */
        {
          const double dth = 0.5 * (t_global - c->tlast[i]);
          double *op = CELL3(c->opos, i), *ov = CELL3(c->ovel, i);
          const double *v = CELL3(c->vel, i);
          for (int a = 0; a < 3; a++) { op[a] = op[a] + (v[a] + ov[a]) * dth; ov[a] = v[a]; }
        }
        c->tlast[i] = c->dt_tick * (double)c->tsysU;
        c->tend[i] = c->dt_tick * (double)c->tsysU + get_dt(c, c->rung[i]);
      } else if (!(c->tlast[i] == t_global)) {
        if (tendi[i] - tl[i] < c->tend[i] - c->tlast[i]) {
          const int r = rungi[i] < 0 ? -1 - rungi[i] : rungi[i];
          c->rung[i] = r;
          c->tend[i] = tendi[i];
          if (rungi[i] < 0) { double *w = WREC(c, i); memset(w + 10, 0, 40 * sizeof(double)); wreset[i] = 1; }
        }
        if (c->bnd[i] == NO_BOUNDARY) {
          double *d = DU(c, i);
          const double *e = dUi + 14 * (size_t)i;
          for (int k = 0; k < NF; k++) d[k] += e[k];
          d[13] += e[13];
          d[10] = d[10] + e[10]; d[11] = d[11] + e[11]; d[12] = d[12] + e[12];
        }
      }
    }
    free(hash); free(wreset); free(dtl);
  }

  /* ======== distribute_fluid_update_data (MPI/distribute_work.cpp:726-748) == */
  double *Wst = (double *)malloc(10 * (size_t)n * sizeof(double));
  for (int i = 0; i < n; i++)
    if (c->active[i] || c->lngb[i]) to_primitive(UU(c, i), c->volume[i], Wst + 10 * (size_t)i);

  /* ======== compute_update0 (MPI/compute_update.cpp:695-970) ======== */
  /* wrec (import copy) keeps the limiter-scaled gradients; update0 writes t */
  {
    double *dUdt = (double *)calloc(14 * (size_t)n, sizeof(double));
    for (int ff = 0; ff < c->nflist; ff++) {
      const int f = c->flist[ff];
      int i = c->s1[f], j = c->s2[f];
      const double *fn = c->fn + 3 * (size_t)f, *fc = c->fc + 3 * (size_t)f;
      const double area = face_area(fn);
      const double ia = 1.0 / area;
      double nrm[3] = {fn[0] * ia, fn[1] * ia, fn[2] * ia};
      const double *xi = CELL3(c->pos, i);
      double dri[3] = {fc[0] - xi[0], fc[1] - xi[1], fc[2] - xi[2]};
      if (c->bnd[i] != NO_BOUNDARY) {
        int t = i; i = j; j = t;
        for (int a = 0; a < 3; a++) { nrm[a] *= -1.0; dri[a] *= -1.0; }
      }
      if (c->bnd[i] != NO_BOUNDARY) continue;
      const double dsh = dri[0] * nrm[0] + dri[1] * nrm[1] + dri[2] * nrm[2];
      const double *Wi = Wst + 10 * (size_t)i;
      const double *Wj = (c->bnd[j] == NO_BOUNDARY) ? Wst + 10 * (size_t)j : Wi;
      const double *vi = CELL3(c->vel, i), *vj = CELL3(c->vel, j);
      const double vij[3] = {vj[0] + vi[0], vj[1] + vi[1], vj[2] + vi[2]};
      const double dvij[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
      const double fij[3] = {dri[0] - nrm[0] * dsh, dri[1] - nrm[1] * dsh, dri[2] - nrm[2] * dsh};
      const double fdv = dvij[0] * fij[0] + dvij[1] * fij[1] + dvij[2] * fij[2];
      const double ids2 = -0.5 * fdv * ((dsh > 0.0) ? 1.0 / sqr(dsh) : 0.0);
      const double wij[3] = {vij[0] * 0.5 + dri[0] * ids2, vij[1] * 0.5 + dri[1] * ids2, vij[2] * 0.5 + dri[2] * ids2};
      double psi, Bn, flux[NF];
      compute_flux(c, wij, Wi, Wj, c->bnd[j], nrm, &psi, &Bn, flux);
      double *di = dUdt + 14 * (size_t)i, *dj = dUdt + 14 * (size_t)j;
      for (int k = 0; k < NF; k++) { di[k] -= flux[k] * area; dj[k] += flux[k] * area; }
      const double pa = psi * area;
      di[10] = di[10] + nrm[0] * pa; di[11] = di[11] + nrm[1] * pa; di[12] = di[12] + nrm[2] * pa;
      dj[10] = dj[10] - nrm[0] * pa; dj[11] = dj[11] - nrm[1] * pa; dj[12] = dj[12] - nrm[2] * pa;
      di[13] += Bn * area;
      dj[13] -= Bn * area;
    }
    for (int a = 0; a < c->nactive; a++) {
      const int i = c->alist[a];
      if (c->bnd[i] != NO_BOUNDARY) continue;
      const double *dot = dUdt + 14 * (size_t)i;
      const double divB = dot[13];
      const double dPsi[3] = {dot[10], dot[11], dot[12]};
      const double *U0 = UU(c, i);
      double W0[NF];
      to_primitive(U0, c->cvol[i], W0);
      while (U0[MASS] + dot[MASS] * get_dt(c, c->rung[i]) <= 0.0 * U0[MASS]) c->rung[i]++;
      const double dt = get_dt(c, c->rung[i]);
      double *r = wrec + 50 * (size_t)i;
      double Uc[NF];
      for (int k = 0; k < NF; k++) Uc[k] = U0[k] + dot[k] * dt;
      {
        Uc[WBX] -= W0[VELX] * divB * dt;
        Uc[WBY] -= W0[VELY] * divB * dt;
        Uc[WBZ] -= W0[VELZ] * divB * dt;
        const double pres = pressure(c, W0);
        const double B2 = W0[BX] * W0[BX] + W0[BY] * W0[BY] + W0[BZ] * W0[BZ];
        const double dcs2 = gamma * pres + B2;
        const double ch_sig = sqrt(dcs2 / W0[DENS]);
        Uc[WBX] -= dPsi[0] * dt;
        Uc[WBY] -= dPsi[1] * dt;
        Uc[WBZ] -= dPsi[2] * dt;
        Uc[MPSI] -= dcs2 * divB * dt;
        const double cr = 0.5;
        const double l_min = pow(c->cvol[i] / (4.0 * M_PI / 3.0), 1.0 / 3.0);
        Uc[MPSI] *= exp(-cr * ch_sig / l_min * dt);
      }
      double W1[NF];
      to_primitive(Uc, c->cvol[i], W1);
      W1[ETHM] = ethm_update(c, W1, i);
      if (W1[ETHM] <= 0.0) { W1[ETHM] = ethm_from_entropy(c, W1); W1[ETHM] = W0[ETHM]; }
      else W1[ENTR] = entropy_from_ethm(c, W1);
      const double idt = 1.0 / dt;
      for (int k = 0; k < NF; k++) r[40 + k] = (W1[k] - W0[k]) * idt;
      /* Wrec.tlast = -dt is carried by the collect step below */
      tendi[i] = -dt; /* reuse as the "tlast < 0" marker of this cell */
    }
    free(dUdt);
  }
  if (snap) copy_wrec_all(c, wrec, snap->wrec_after_update0);
  if (snap && snap->rung_after_update0) memcpy(snap->rung_after_update0, c->rung, sizeof(int) * n);

  /* ======== compute_reconstruction (MPI/compute_reconstruction.cpp:24-199) == */
  {
    double cl[3 * 64];
    for (int a = 0; a < c->nactive; a++) {
      const int i = c->alist[a];
      double *r = wrec + 50 * (size_t)i;
      const double *Wi = Wst + 10 * (size_t)i;
      if (c->bnd[i] != NO_BOUNDARY) {
        memcpy(r, Wi, 10 * sizeof(double));
        memset(r + 10, 0, 40 * sizeof(double));
        continue;
      }
      double Wx[NF] = {0}, Wy[NF] = {0}, Wz[NF] = {0}, mn[NF] = {0}, mx[NF] = {0};
      const double *ip = CELL3(c->pos, i);
      int zero_flag = 0;
      double sc[3] = {0.0, 0.0, 0.0};
      const int nfc = (int)(c->off[i + 1] - c->off[i]);
      double *cent = nfc <= 64 ? cl : (double *)malloc(3 * sizeof(double) * nfc);
      for (int q = 0; q < nfc; q++) {
        const int f = c->ids[c->off[i] + q];
        const double *fc = c->fc + 3 * (size_t)f, *fn = c->fn + 3 * (size_t)f;
        double d[3];
        for (int a3 = 0; a3 < 3; a3++) {
          d[a3] = fc[a3] - ip[a3];
          const double L = c->p.box[a3];
          if (d[a3] > 0.5 * L) d[a3] -= L;
          else if (d[a3] < -0.5 * L) d[a3] += L;
        }
        cent[3 * q] = d[0]; cent[3 * q + 1] = d[1]; cent[3 * q + 2] = d[2];
        sc[0] = sc[0] + d[0]; sc[1] = sc[1] + d[1]; sc[2] = sc[2] + d[2];
        const double area = face_area(fn);
        const double s = ((d[0] * fn[0] + d[1] * fn[1] + d[2] * fn[2]) < 0.0) ? (-1.0 / area) : (1.0 / area);
        const double nrm[3] = {fn[0] * s, fn[1] * s, fn[2] * s};
        const double dsh = d[0] * nrm[0] + d[1] * nrm[1] + d[2] * nrm[2];
        const double ids = (dsh != 0.0) ? 0.5 / dsh : 0.0;
        const double idsA = area * ids;
        const double drh[3] = {nrm[0] * dsh, nrm[1] * dsh, nrm[2] * dsh};
        const double fij[3] = {d[0] - drh[0], d[1] - drh[1], d[2] - drh[2]};
        const int j = ngb_of(c, f, i);
        if (c->bnd[j] != NO_BOUNDARY) { zero_flag = 1; break; }
        const double *Wj = Wst + 10 * (size_t)j;
        for (int k = 0; k < NF; k++) {
          const double sum = Wj[k] + Wi[k];
          const double diff = Wj[k] - Wi[k];
          mn[k] = dmin(mn[k], diff);
          mx[k] = dmax(mx[k], diff);
          Wx[k] += (sum * drh[0] + diff * fij[0]) * idsA;
          Wy[k] += (sum * drh[1] + diff * fij[1]) * idsA;
          Wz[k] += (sum * drh[2] + diff * fij[2]) * idsA;
        }
      }
      if (zero_flag) {
        memcpy(r, Wi, 10 * sizeof(double));
        memset(r + 10, 0, 40 * sizeof(double));
        if (cent != cl) free(cent);
        continue;
      }
      const double invV = 1.0 / c->cvol[i];
      for (int k = 0; k < NF; k++) { Wx[k] *= invV; Wy[k] *= invV; Wz[k] *= invV; }
      double lm[NF];
      for (int k = 0; k < NF; k++) lm[k] = 1.0;
      const double sum_dt = get_dt(c, c->rung[i]);
      for (int q = 0; q < nfc; q++)
        for (int k = 0; k < NF; k++) {
          const double dWx = Wx[k] * cent[3 * q] + Wy[k] * cent[3 * q + 1] + Wz[k] * cent[3 * q + 2];
          lm[k] = dmin(lm[k], limiter(dWx, mn[k], mx[k]));
        }
      if (cent != cl) free(cent);
      for (int k = 0; k < NF; k++) {
        const double tau = lm[k];
        Wx[k] *= tau; Wy[k] *= tau; Wz[k] *= tau;
        r[40 + k] *= tau;
        r[k] = Wi[k];
        r[10 + k] = Wx[k]; r[20 + k] = Wy[k]; r[30 + k] = Wz[k];
      }
      {
        const int k = DENS;
        const double dWx = Wx[k] * sc[0] + Wy[k] * sc[1] + Wz[k] * sc[2];
        const double dWp = dWx + r[40 + k] * sum_dt;
        const double dW = dmax(dWx, dWp);
        if (dW > 0.0) {
          const double alpha = dmin(1.0, 0.9 * Wi[k] / dW);
          r[10 + k] *= alpha; r[20 + k] *= alpha; r[30 + k] *= alpha; r[40 + k] *= alpha;
        }
      }
    }
  }
  if (snap) copy_wrec_all(c, wrec, snap->wrec_after_recon);

  /* ======== collect_reconstruction (MPI/distribute_work.cpp:807-835) ====== */
  for (int a = 0; a < c->nactive; a++) {
    const int i = c->alist[a];
    memcpy(WREC(c, i), wrec + 50 * (size_t)i, 50 * sizeof(double));
    if (c->bnd[i] == NO_BOUNDARY) { /* tlast = -dt was set by compute_update0 */
      const double tln = tendi[i];
      if (tln < 0.0) {
        c->rung[i] = imax(c->rung[i], get_rung(c, -tln));
        c->tend[i] = t_global + get_dt(c, c->rung[i]);
      }
    }
  }
  if (shared) {
    int rmax = 0;
    for (int a = 0; a < c->nactive; a++) rmax = imax(rmax, c->rung[c->alist[a]]);
    for (int a = 0; a < c->nactive; a++) {
      c->rung[c->alist[a]] = rmax;
      c->tend[c->alist[a]] = t_global + get_dt(c, rmax);
    }
  }

  free(Wst); free(failed); free(wrec); free(dUi); free(Ui); free(rungi); free(tendi);
  free(voli); free(veli);
  return c->nactive;
}

int fvo_compute_flux(const fvo_ctx *c, int nface, const double *wij, const double *Wi,
                     const double *Wj, const int *jbnd, const double *normal, double *psi,
                     double *Bn, double *flux) {
  for (int f = 0; f < nface; f++)
    compute_flux(c, wij + 3 * (size_t)f, Wi + 10 * (size_t)f, Wj + 10 * (size_t)f, jbnd ? jbnd[f] : 0,
                 normal + 3 * (size_t)f, psi + f, Bn + f, flux + 10 * (size_t)f);
  return 0;
}
