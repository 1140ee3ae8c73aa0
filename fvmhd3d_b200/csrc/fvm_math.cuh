// Device math of the fvmhd3d fluid hot path: primitive/conservative
// conversion, EOS hooks, the rotated-frame face flux with the moving-face
// HLLD Riemann solver, and the slope limiter.  Every function keeps the
// reference's operation order (file:line cited per function); the only
// systematic difference from the CPU build is fused multiply-add
// contraction, which moves results by a few ulps.
#pragma once
#include <cstdint>

namespace fvm {

enum { NF = 10 };
enum { MASS = 0, MOMX, MOMY, MOMZ, ENER, WBX, WBY, WBZ, MPSI, MENTR };
enum { DENS = 0, VELX, VELY, VELZ, ETHM, BX, BY, BZ, PSI, ENTR };
enum { NO_BOUNDARY = 0, REFLECTING = 1, OUTFLOW = 2, DIOD = 3 };
enum { RUNGMAX = 32 };

// The reference uses the legacy SVID constant HUGE (a float) in its timestep
// formulas (MPI/compute_timestep.cpp:27,44,81).
#define FVM_HUGE ((double)3.40282347e+38F)

struct Params {
  double gamma, courant;
  double box[3];
  double dtmax, dt_tick;
  int eos;              // 0 ideal gas, 1 isothermal disk
  double iso_GM, iso_cfac;
  int static_mesh;      // 1: compute_pvel1 hook with vel = 0 (static generators)
  // per cell: (V / (4 pi / 3))^(1/3), the length of the CFL timestep and of
  // the Dedner damping, computed once per mesh (a cell's volume changes only
  // with its mesh)
  const double *hcell;
  // per cell, or null: the cell is a copy of another rank's cell, left out
  // of the timestep minimum (fvm_set_halo)
  const unsigned char *halo;
};

template <typename T> __host__ __device__ __forceinline__ T sqr(T x) { return x * x; }
// std::min / std::max semantics (first argument wins ties)
template <typename T> __host__ __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T> __host__ __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }

// ---- scheduler arithmetic (MPI/Scheduler.h:33-38, 87-104) ----------------
__host__ __device__ __forceinline__ int exp_of(double dt) {
#ifdef __CUDA_ARCH__
  const unsigned long long u = (unsigned long long)__double_as_longlong(dt);
#else
  unsigned long long u;
  __builtin_memcpy(&u, &dt, 8);
#endif
  return (int)((u >> 52) & 0xfff);
}
__host__ __device__ __forceinline__ double get_dt(const Params &P, int rung) {
  const unsigned long long dtU = 1ULL << (RUNGMAX - 1 - rung);
  return P.dt_tick * (double)dtU;
}
__host__ __device__ __forceinline__ int get_rung(const Params &P, double dt, int min_rung) {
  const int r = exp_of(P.dtmax) - exp_of(dt);
  return r < min_rung ? min_rung : r;
}

// ---- EOS hooks (ideal gas MPI/set_problem.cpp:123-137; isothermal disk
//      MPI/problems/mri_disk3d.cpp:368-389) ------------------------------
template <typename T>
__host__ __device__ __forceinline__ T pressure(const Params &P, const T *W) {
  if (P.eos == 0) return P.gamma > 1.0 ? T(P.gamma - 1.0) * W[ETHM] : W[ETHM];
  return W[ETHM];
}
template <typename T>
__device__ __forceinline__ T entropy_from_ethm(const Params &P, const T *W) {
  if (P.eos == 0) return T(P.gamma - 1.0) * W[ETHM] / pow(W[DENS], T(P.gamma));
  return T(1.0);
}
template <typename T>
__device__ __forceinline__ T ethm_from_entropy(const Params &P, const T *W) {
  if (P.eos == 0) return W[ENTR] * pow(W[DENS], T(P.gamma)) / T(P.gamma - 1.0);
  return T(-1.0);
}
__device__ __forceinline__ double ethm_update(const Params &P, const double *W, const double *pos) {
  if (P.eos == 0) return W[ETHM];
  const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  return (P.iso_GM / r) * sqr(P.iso_cfac) * W[DENS];
}

// ---- prim <-> cons (MPI/Fluid.h:55-129) ----------------------------------
template <typename T>
__host__ __device__ __forceinline__ void to_primitive(const T *U, T V, T *W) {
  const T iM = T(1.0) / U[MASS];
  const T iV = T(1.0) / V;
  W[DENS] = U[MASS] * iV;
  W[VELX] = U[MOMX] * iM;
  W[VELY] = U[MOMY] * iM;
  W[VELZ] = U[MOMZ] * iM;
  W[BX] = U[WBX] * iV;
  W[BY] = U[WBY] * iV;
  W[BZ] = U[WBZ] * iV;
  W[PSI] = U[MPSI] * iM;
  W[ENTR] = U[MENTR] * iM;
  W[ETHM] = U[ENER] * iV - T(0.5) * (sqr(W[BX]) + sqr(W[BY]) + sqr(W[BZ])) -
            T(0.5) * (sqr(W[VELX]) + sqr(W[VELY]) + sqr(W[VELZ])) * W[DENS];
}
template <typename T>
__device__ __forceinline__ void to_conservative(const T *W, T V, T *U) {
  const T M = W[DENS] * V;
  U[MASS] = W[DENS] * V;
  U[MOMX] = W[VELX] * M;
  U[MOMY] = W[VELY] * M;
  U[MOMZ] = W[VELZ] * M;
  U[WBX] = W[BX] * V;
  U[WBY] = W[BY] * V;
  U[WBZ] = W[BZ] * V;
  U[MPSI] = W[PSI] * M;
  U[MENTR] = W[ENTR] * M;
  U[ENER] = W[ETHM] * V + T(0.5) * (sqr(W[BX]) + sqr(W[BY]) + sqr(W[BZ])) * V +
            T(0.5) * (sqr(W[VELX]) + sqr(W[VELY]) + sqr(W[VELZ])) * M;
}

// ---- HLLD at face speed w (MPI/compute_update.cpp:1109-1341) -------------
// Outputs the 8 rotated-frame fluxes MASS, MOMX..Z, ENER, WBX..Z.
template <typename T>
__device__ __forceinline__ void riemann_hlld(T gamma, T *flux, T Bx, T w, T dens_L, T pres_L,
                                             T ethm_L, T velx_L, T vely_L, T velz_L, T By_L,
                                             T Bz_L, T dens_R, T pres_R, T ethm_R, T velx_R,
                                             T vely_R, T velz_R, T By_R, T Bz_R) {
  const T signBx = Bx == T(0) ? T(0) : (Bx > T(0) ? T(1) : T(-1));
  const T momx_L = dens_L * velx_L, momy_L = dens_L * vely_L, momz_L = dens_L * velz_L;
  const T momx_R = dens_R * velx_R, momy_R = dens_R * vely_R, momz_R = dens_R * velz_R;
  const T chalf = T(0.5);
  const T B2_L = sqr(Bx) + sqr(By_L) + sqr(Bz_L);
  const T v2_L = sqr(velx_L) + sqr(vely_L) + sqr(velz_L);
  const T etot_L = ethm_L + chalf * (dens_L * v2_L + B2_L);
  const T B2_R = sqr(Bx) + sqr(By_R) + sqr(Bz_R);
  const T v2_R = sqr(velx_R) + sqr(vely_R) + sqr(velz_R);
  const T etot_R = ethm_R + chalf * (dens_R * v2_R + B2_R);
  const T gpbl = gamma * pres_L + B2_L, gpbr = gamma * pres_R + B2_R;
  const T cfl2 = gpbl / dens_L, cfr2 = gpbr / dens_R;
  const T cfmax = sqrt(smax(cfl2, cfr2));
  const T S_L = smin(velx_L, velx_R) - cfmax;
  const T S_R = smax(velx_L, velx_R) + cfmax;
  const T pT_L = pres_L + chalf * B2_L, pT_R = pres_R + chalf * B2_R;
  // iSM and ipTs are the same quantity in the reference (lines 1157,1161)
  const T iSM = T(1) / ((S_R - velx_R) * dens_R - (S_L - velx_L) * dens_L);
  const T S_M = iSM * ((S_R - velx_R) * momx_R - (S_L - velx_L) * momx_L - pT_R + pT_L);
  const T pT_s = iSM * ((S_R - velx_R) * dens_R * pT_L - (S_L - velx_L) * dens_L * pT_R +
                        dens_L * dens_R * (S_R - velx_R) * (S_L - velx_L) * (velx_R - velx_L));
  const T B2x = Bx * Bx;
  const T iSLmSM = T(1) / (S_L - S_M), iSRmSM = T(1) / (S_R - S_M);
  const T dens_L_s = dens_L * (S_L - velx_L) * iSLmSM;
  const T dens_R_s = dens_R * (S_R - velx_R) * iSRmSM;
  const T divL = dens_L * (S_L - velx_L) * (S_L - S_M) - B2x;
  const T divR = dens_R * (S_R - velx_R) * (S_R - S_M) - B2x;
  const T idivL = (divL != T(0)) ? T(1) / divL : T(0);
  const T idivR = (divR != T(0)) ? T(1) / divR : T(0);
  const T vely_L_s = vely_L - Bx * By_L * (S_M - velx_L) * idivL;
  const T velz_L_s = velz_L - Bx * Bz_L * (S_M - velx_L) * idivL;
  const T By_L_s = By_L * (dens_L * sqr(S_L - velx_L) - B2x) * idivL;
  const T Bz_L_s = Bz_L * (dens_L * sqr(S_L - velx_L) - B2x) * idivL;
  const T vely_R_s = vely_R - Bx * By_R * (S_M - velx_R) * idivR;
  const T velz_R_s = velz_R - Bx * Bz_R * (S_M - velx_R) * idivR;
  const T By_R_s = By_R * (dens_R * sqr(S_R - velx_R) - B2x) * idivR;
  const T Bz_R_s = Bz_R * (dens_R * sqr(S_R - velx_R) - B2x) * idivR;
  const T vB_L = velx_L * Bx + vely_L * By_L + velz_L * Bz_L;
  const T vB_L_s = S_M * Bx + vely_L_s * By_L_s + velz_L_s * Bz_L_s;
  const T etot_L_s = ((S_L - velx_L) * etot_L - pT_L * velx_L + pT_s * S_M + Bx * (vB_L - vB_L_s)) * iSLmSM;
  const T vB_R = velx_R * Bx + vely_R * By_R + velz_R * Bz_R;
  const T vB_R_s = S_M * Bx + vely_R_s * By_R_s + velz_R_s * Bz_R_s;
  const T etot_R_s = ((S_R - velx_R) * etot_R - pT_R * velx_R + pT_s * S_M + Bx * (vB_R - vB_R_s)) * iSRmSM;
  const T sDens_L_s = sqrt(dens_L_s), sDens_R_s = sqrt(dens_R_s);
  const T S_L_s = S_M - fabs(Bx / sDens_L_s);
  const T S_R_s = S_M + fabs(Bx / sDens_R_s);
  const T idsqroot = T(1) / (sDens_L_s + sDens_R_s);
  const T vely_ss = idsqroot * (sDens_L_s * vely_L_s + sDens_R_s * vely_R_s + (By_R_s - By_L_s) * signBx);
  const T velz_ss = idsqroot * (sDens_L_s * velz_L_s + sDens_R_s * velz_R_s + (Bz_R_s - Bz_L_s) * signBx);
  const T By_ss = idsqroot * (sDens_L_s * By_R_s + sDens_R_s * By_L_s + sDens_L_s * sDens_R_s * (vely_R_s - vely_L_s) * signBx);
  const T Bz_ss = idsqroot * (sDens_L_s * Bz_R_s + sDens_R_s * Bz_L_s + sDens_L_s * sDens_R_s * (velz_R_s - velz_L_s) * signBx);
  const T vB_ss = S_M * Bx + vely_ss * By_ss + velz_ss * Bz_ss;
  const T etot_L_ss = etot_L_s - sDens_L_s * (vB_L_s - vB_ss) * signBx;
  const T etot_R_ss = etot_R_s + sDens_R_s * (vB_R_s - vB_ss) * signBx;

  const bool w_lt_SL = w <= S_L, w_le_SLs = w <= S_L_s, w_le_SM = w <= S_M;
  const bool w_le_SRs = w <= S_R_s, w_le_SR = w <= S_R;
  // region coefficients: F = F_side + a U** + b U* + c U
  const T a = w_le_SLs ? T(0) : (w_le_SM ? S_L_s - w : (w_le_SRs ? S_R_s - w : T(0)));
  const T b = w_lt_SL ? T(0)
            : (w_le_SLs ? +S_L - w
            : (w_le_SM ? -S_L_s + S_L
            : (w_le_SRs ? -S_R_s + S_R : (w_le_SR ? +S_R - w : T(0)))));
  const T c = w_lt_SL ? -w : (w_le_SLs ? -S_L : (w_le_SM ? -S_L : (w_le_SRs ? -S_R : (w_le_SR ? -S_R : -w))));
  // side selection before the flux sums (only one side's values are live)
  const T dens = w_le_SM ? dens_L : dens_R;
  const T dens_s = w_le_SM ? dens_L_s : dens_R_s;
  const T velx = w_le_SM ? velx_L : velx_R;
  const T vely = w_le_SM ? vely_L : vely_R;
  const T velz = w_le_SM ? velz_L : velz_R;
  const T by = w_le_SM ? By_L : By_R;
  const T bz = w_le_SM ? Bz_L : Bz_R;
  const T pT = w_le_SM ? pT_L : pT_R;
  const T vB = w_le_SM ? vB_L : vB_R;
  const T mx = w_le_SM ? momx_L : momx_R;
  const T my = w_le_SM ? momy_L : momy_R;
  const T mz = w_le_SM ? momz_L : momz_R;
  const T etot = w_le_SM ? etot_L : etot_R;
  const T etot_s = w_le_SM ? etot_L_s : etot_R_s;
  const T etot_ss = w_le_SM ? etot_L_ss : etot_R_ss;
  const T vy_s = w_le_SM ? vely_L_s : vely_R_s;
  const T vz_s = w_le_SM ? velz_L_s : velz_R_s;
  const T by_s = w_le_SM ? By_L_s : By_R_s;
  const T bz_s = w_le_SM ? Bz_L_s : Bz_R_s;
  const T fdens = dens * velx;
  const T fmomx = mx * velx + pT - B2x;
  const T fmomy = my * velx - Bx * by;
  const T fmomz = mz * velx - Bx * bz;
  const T fetot = etot * velx + pT * velx - Bx * vB;
  const T fby = by * velx - Bx * vely;
  const T fbz = bz * velx - Bx * velz;
  flux[MASS] = fdens + a * dens_s + b * dens_s + c * dens;
  flux[ENER] = fetot + a * etot_ss + b * etot_s + c * etot;
  flux[MOMX] = fmomx + a * (dens_s * S_M) + b * (dens_s * S_M) + c * mx;
  flux[MOMY] = fmomy + a * (dens_s * vely_ss) + b * (dens_s * vy_s) + c * my;
  flux[MOMZ] = fmomz + a * (dens_s * velz_ss) + b * (dens_s * vz_s) + c * mz;
  flux[WBY] = fby + a * By_ss + b * by_s + c * by;
  flux[WBZ] = fbz + a * Bz_ss + b * bz_s + c * bz;
  flux[WBX] = -w * Bx;
}

// ---- rotated-frame face flux (MPI/compute_update.cpp:973-1095) -----------
// Wi/Wj primitive face states, normal the unit normal i->j, wij the face
// velocity.  Returns the 10 lab-frame fluxes, psi_ij and Bn_ij.
// The exact Riemann solver as a compute_flux hook.
struct HlldSolver {
  template <typename T>
  __device__ __forceinline__ bool operator()(T gamma, T *F, T Bx, T w, T dens_L, T pres_L, T ethm_L, T velx_L,
                                             T vely_L, T velz_L, T By_L, T Bz_L, T dens_R, T pres_R, T ethm_R,
                                             T velx_R, T vely_R, T velz_R, T By_R, T Bz_R, T chL, T chR,
                                             int jbnd) {
    riemann_hlld<T>(gamma, F, Bx, w, dens_L, pres_L, ethm_L, velx_L, vely_L, velz_L, By_L, Bz_L, dens_R, pres_R,
                    ethm_R, velx_R, vely_R, velz_R, By_R, Bz_R);
    return true;
  }
};

// compute_flux with the rotated-frame Riemann solve delegated to `solve`
// (which may decline: then nothing after psi_ij / Bn_ij is computed and
// false is returned).
template <typename T, typename Solver>
__device__ __forceinline__ bool compute_flux_with(const Params &P, const T *wij, const T *Wi, const T *Wj,
                                                  int jbnd, const T *normal, T &psi_ij, T &Bn_ij, T *flux,
                                                  Solver &solve) {
  const T gamma = T(P.gamma);
  const T ex = normal[0], ey = normal[1], ez = normal[2];
  const T ds = sqrt(ex * ex + ey * ey);
  const T ids = (ds != T(0)) ? T(1) / ds : T(0);
  const T cosph = (ids == T(0)) ? T(1) : ex * ids;
  const T sinph = (ids == T(0)) ? T(0) : ey * ids;
  const T costh = ez, sinth = ds;
  const T Axx = cosph * sinth, Axy = sinth * sinph, Axz = costh;
  const T Ayx = -sinph, Ayy = cosph;
  const T Azx = -costh * cosph, Azy = -costh * sinph, Azz = sinth;
  const T dens_L = Wi[DENS], ethm_L = Wi[ETHM];
  const T velx_L = Axx * Wi[VELX] + Axy * Wi[VELY] + Axz * Wi[VELZ];
  const T vely_L = Ayx * Wi[VELX] + Ayy * Wi[VELY];
  const T velz_L = Azx * Wi[VELX] + Azy * Wi[VELY] + Azz * Wi[VELZ];
  const T Bx_L = Axx * Wi[BX] + Axy * Wi[BY] + Axz * Wi[BZ];
  const T By_L = Ayx * Wi[BX] + Ayy * Wi[BY];
  const T Bz_L = Azx * Wi[BX] + Azy * Wi[BY] + Azz * Wi[BZ];
  const T psiL = Wi[PSI], entrL = Wi[ENTR];
  const T dens_R = Wj[DENS], ethm_R = Wj[ETHM];
  T velx_R = Axx * Wj[VELX] + Axy * Wj[VELY] + Axz * Wj[VELZ];
  const T vely_R = Ayx * Wj[VELX] + Ayy * Wj[VELY];
  const T velz_R = Azx * Wj[VELX] + Azy * Wj[VELY] + Azz * Wj[VELZ];
  const T Bx_R = Axx * Wj[BX] + Axy * Wj[BY] + Axz * Wj[BZ];
  const T By_R = Ayx * Wj[BX] + Ayy * Wj[BY];
  const T Bz_R = Azx * Wj[BX] + Azy * Wj[BY] + Azz * Wj[BZ];
  const T psiR = Wj[PSI], entrR = Wj[ENTR];
  const T pres_L = pressure(P, Wi), pres_R = pressure(P, Wj);
  const T wn_ij = Axx * wij[0] + Axy * wij[1] + Axz * wij[2];
  if (jbnd == REFLECTING) velx_R = -velx_R;
  else if (jbnd == DIOD) velx_R = smax(velx_R - T(1.2) * wn_ij, T(0)) + T(1.2) * wn_ij;
  const T cfl2 = (gamma * pres_L + sqr(Bx_L) + sqr(By_L) + sqr(Bz_L)) / dens_L;
  const T cfr2 = (gamma * pres_R + sqr(Bx_R) + sqr(By_R) + sqr(Bz_R)) / dens_R;
  const T chL = sqrt(cfl2), chR = sqrt(cfr2);
  const T ich = T(1) / (chL + chR);
  Bn_ij = (Bx_L * chL + Bx_R * chR + (psiL - psiR)) * ich;
  psi_ij = (psiL * chR + psiR * chL + chR * chL * (Bx_L - Bx_R)) * ich;
  T F[8];
  if (!solve(gamma, F, Bn_ij, wn_ij, dens_L, pres_L, ethm_L, velx_L, vely_L, velz_L, By_L, Bz_L, dens_R, pres_R,
             ethm_R, velx_R, vely_R, velz_R, By_R, Bz_R, chL, chR, jbnd))
    return false;
  // back-rotation with the transpose of A
  flux[MASS] = F[MASS];
  flux[ENER] = F[ENER];
  flux[MOMX] = Axx * F[MOMX] + Ayx * F[MOMY] + Azx * F[MOMZ];
  flux[MOMY] = Axy * F[MOMX] + Ayy * F[MOMY] + Azy * F[MOMZ];
  flux[MOMZ] = Axz * F[MOMX] + Azz * F[MOMZ];
  flux[WBX] = Axx * F[WBX] + Ayx * F[WBY] + Azx * F[WBZ];
  flux[WBY] = Axy * F[WBX] + Ayy * F[WBY] + Azy * F[WBZ];
  flux[WBZ] = Axz * F[WBX] + Azz * F[WBZ];
  flux[MPSI] = F[MASS] * (F[MASS] > T(0) ? psiL : psiR);
  flux[MENTR] = F[MASS] * (F[MASS] > T(0) ? entrL : entrR);
  return true;
}

template <typename T>
__device__ __forceinline__ void compute_flux(const Params &P, const T *wij, const T *Wi, const T *Wj,
                                             int jbnd, const T *normal, T &psi_ij, T &Bn_ij, T *flux) {
  HlldSolver exact;
  compute_flux_with<T>(P, wij, Wi, Wj, jbnd, normal, psi_ij, Bn_ij, flux, exact);
}

// ---- limiter (MPI/compute_reconstruction.cpp:5-22) -----------------------
template <typename T>
__device__ __forceinline__ T Phi(T x) {
  const T e = T(0.2 * 1.0e-16);
  return (x * x + T(2) * x + e) / (x * x + x + T(2) + e);
}
// Branch-free form: both candidate ratios share one division, and the
// threshold test selects the result, so a warp never splits on the sign of
// dWi.  The selected value is the one the reference's branches compute.
template <typename T>
__device__ __forceinline__ T limiter(T dWi, T dWj_min, T dWj_max) {
  const bool flat = fabs(dWi) <= T(1.0e-16) * smax(fabs(dWj_max), fabs(dWj_min));
  const T num = dWi < T(0) ? dWj_min : dWj_max;
  const T den = flat ? T(1) : dWi;
  const T phi = Phi(num / den);
  return flat ? T(1) : phi;
}

// Running minimum of the limiter over a cell's faces, with no division per
// face.  Phi is increasing on [0, 2] (its derivative has the sign of
// 4 + 4x - x^2 + e) and Phi(x) >= 1 exactly when x >= 2, so
// min(1, min over faces of Phi(x_f)) = Phi(min(2, min over faces of x_f)),
// a flat face counting as x_f = 2.  x_f = num/dWi >= 0 (num has the sign of
// dWi) is kept as the fraction bn/bd = |num|/|dWi|, compared by
// cross-multiplication; the caller starts from bn = 2, bd = 1 and ends with
// limiter_finish, one evaluation of Phi.  thr = limiter_thr(min, max) is the
// reference's flatness threshold, fixed over the face loop.  Where two faces'
// ratios differ by less than rounding, the face kept may differ from the
// reference's running minimum of rounded Phi values by a few units in the
// last place.
template <typename T>
__device__ __forceinline__ T limiter_thr(T dWj_min, T dWj_max) {
  return T(1.0e-16) * smax(fabs(dWj_max), fabs(dWj_min));
}
template <typename T>
__device__ __forceinline__ void limiter_ratio(T &bn, T &bd, T dWi, T dWj_min, T dWj_max, T thr) {
  const T a = fabs(dWi < T(0) ? dWj_min : dWj_max), b = fabs(dWi);
  if (b > thr && a * bd < bn * b) { bn = a; bd = b; }
}
template <typename T>
__device__ __forceinline__ T limiter_finish(T bn, T bd) {
  if (!(bn < T(2) * bd)) return T(1);
  const T phi = Phi(bn / bd);
  return phi < T(1) ? phi : T(1);
}

}  // namespace fvm
