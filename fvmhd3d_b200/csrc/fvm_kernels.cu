// sm_100a kernels of the fvmhd3d fluid hot path and the C-ABI context
// (include/fvmhd3d_b200.h).
//
// Data layout in HBM (one record per cell / face, 16-byte aligned):
//   faces  s12 int2, geo double4 (unit normal, area), cen double4 (centroid)
//   cells  U double[10], dU double[14], Wrec double[50] (w,x,y,z,t),
//          pos/vel double[3], tlast/tend/volp double, rung/bnd int,
//          CSR off[n+1] / lnk[] of face ids (cell face order of the mesh)
//
// Stage kernels follow the reference call sequence (MPI/iterate.cpp:95-113).
// Per-cell reductions over faces (limiter min/max, tau, gradients, timestep,
// flux sums) are gathers in the cell's face order, so every run gives the
// same bits.  Each face flux is evaluated once by a face-parallel kernel that
// stores the face's contribution; the owning cells then gather it.
#include "fvm_math.cuh"
#include "../../include/fvmhd3d_b200.h"

#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <string>

using namespace fvm;

namespace {

enum : unsigned char { A_ACTIVE = 1, A_LNGB = 2, A_HASNGB = 4 };
enum : unsigned char { F_SWAP = 1, F_SKIPJ = 2, F_OFF = 4 };

struct Dev {
  // mesh
  int2 *s12;
  double4 *geo, *cen;
  double *cvol, *ccen;
  int *off, *lnk;
  // state
  double *pos, *vel, *tlast, *tend, *volp;
  int *rung, *bnd;
  double *U, *dU, *Wrec;
  // per-step work
  unsigned char *act0, *act, *hash, *fcode, *fcode2;
  double *tau, *fcon, *fcon2, *Wst, *dtl, *stepdU;
  // scalars: dmin (double), ints [maxrung, nactive], counters
  double *dscal;
  int *iscal;
  unsigned long long *counters;
};

__device__ __forceinline__ bool face_active(const unsigned char *act, const int *bnd, int a, int b) {
  return ((act[a] & A_ACTIVE) && bnd[a] == NO_BOUNDARY) || ((act[b] & A_ACTIVE) && bnd[b] == NO_BOUNDARY);
}

__device__ __forceinline__ void ld3(const double *p, double *o) { o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; }

// ---- begin_step: active flags (Scheduler::pull_active_list) ---------------
__global__ void k_active(int n, const int *__restrict__ rung, unsigned long long flags,
                         unsigned char *__restrict__ act0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rung[i];
  act0[i] = (r >= 0 && r < RUNGMAX && ((flags >> (RUNGMAX - 1 - r)) & 1ULL)) ? A_ACTIVE : 0;
}

// site flags of build_mesh_active (MPI/build_mesh_active.cpp:524-528)
__global__ void k_ngbflags(int n, const int *__restrict__ off, const int *__restrict__ lnk,
                           const int2 *__restrict__ s12, const unsigned char *__restrict__ act0,
                           unsigned char *__restrict__ act, int *__restrict__ iscal) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool ai = act0[i] & A_ACTIVE;
  bool other = false;
  for (int q = off[i]; q < off[i + 1]; q++) {
    const int2 e = s12[lnk[q]];
    const int j = e.x == i ? e.y : e.x;
    const bool aj = act0[j] & A_ACTIVE;
    if (ai != aj) { other = true; break; }
  }
  unsigned char f = ai ? A_ACTIVE : 0;
  if (ai && other) f |= A_HASNGB;
  if (!ai && other) f |= A_LNGB;
  act[i] = f;
  if (ai) atomicAdd(&iscal[1], 1);
}

// ---- slope_limiter (MPI/compute_reconstruction.cpp:201-602) --------------
// Two threads per imported cell, each owning five of the ten primitives: face
// pass 1 (min/max of neighbour differences) and face pass 2 (limiter of the
// space+time extrapolated difference) over the cell's active faces.  The
// result tau is applied on the fly by the corrector, so Wrec is not modified.
constexpr int KH = 5;  // primitives per thread in the two-threads-per-cell kernels

__global__ void __launch_bounds__(128) k_limiter(int n, Params P, double t_global,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ s12,
    const double4 *__restrict__ geo, const double4 *__restrict__ cen,
    const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ tlast,
    const double *__restrict__ Wrec, double *__restrict__ tau) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t >> 1);
  const int k0 = (int)(t & 1) * KH;
  if (i >= n) return;
  if (!(act[i] & (A_ACTIVE | A_LNGB))) return;
  const double *ri = Wrec + 50 * (size_t)i + k0;
  double mn[KH], mx[KH], ln[KH], lq[KH], wi[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { mn[k] = 0.0; mx[k] = 0.0; ln[k] = 1.0; lq[k] = 1.0; wi[k] = ri[k]; }
  const int q0 = off[i], q1 = off[i + 1];
  bool zero = false;
  for (int q = q0; q < q1; q++) {
    const int f = lnk[q];
    const int2 e = s12[f];
    if (!face_active(act, bnd, e.x, e.y)) continue;
    if (bnd[e.x] != NO_BOUNDARY || bnd[e.y] != NO_BOUNDARY) { zero = true; continue; }
    const int j = e.x == i ? e.y : e.x;
    const double *rj = Wrec + 50 * (size_t)j + k0;
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const double diff = rj[k] - wi[k];
      mn[k] = smin(mn[k], diff);
      mx[k] = smax(mx[k], diff);
    }
  }
  double *to = tau + 10 * (size_t)i + k0;
  if (zero) {
#pragma unroll
    for (int k = 0; k < KH; k++) to[k] = 0.0;
    return;
  }
  double gx[KH], gy[KH], gz[KH], gt[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { gx[k] = ri[10 + k]; gy[k] = ri[20 + k]; gz[k] = ri[30 + k]; gt[k] = ri[40 + k]; }
  for (int q = q0; q < q1; q++) {
    const int f = lnk[q];
    const int2 e = s12[f];
    if (!face_active(act, bnd, e.x, e.y)) continue;
    const double dtI = t_global - tlast[e.x], dtJ = t_global - tlast[e.y];
    const double dth = 0.5 * smin(dtI, dtJ);
    const double4 g = geo[f], c = cen[f];
    const double *pa = pos + 3 * (size_t)e.x;
    const double dri[3] = {c.x - pa[0], c.y - pa[1], c.z - pa[2]};
    const double dsh = dri[0] * g.x + dri[1] * g.y + dri[2] * g.z;
    const bool own = e.x == i;
    const double dsl = own ? 0.0 : 2.0 * dsh;
    const double dr[3] = {dri[0] - g.x * dsl, dri[1] - g.y * dsl, dri[2] - g.z * dsl};
    const double dtt = own ? dtI - dth : dtJ - dth;
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const double dWx = gx[k] * dr[0] + gy[k] * dr[1] + gz[k] * dr[2];
      const double dW = dWx + gt[k] * dtt;
      limiter_min(ln[k], lq[k], dW, mn[k], mx[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < KH; k++) to[k] = ln[k] / lq[k];
}

// ---- compute_update face pass (MPI/compute_update.cpp:106-269) -----------
// One thread per face: half-step extrapolated face states, face velocity,
// rotated-frame HLLD flux.  Stores flux*dt*area, gradPsi and divB
// contributions for the owning cells to gather.
__global__ void __launch_bounds__(128) k_corr_flux(int nf, Params P, double t_global,
    const int2 *__restrict__ s12, const double4 *__restrict__ geo, const double4 *__restrict__ cen,
    const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ vel, const double *__restrict__ tlast,
    const double *__restrict__ Wrec, const double *__restrict__ tau,
    double *__restrict__ fcon, unsigned char *__restrict__ fcode) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int2 e = s12[f];
  if (!face_active(act, bnd, e.x, e.y)) { fcode[f] = F_OFF; return; }
  int i = e.x, j = e.y;
  const double4 g = geo[f], c = cen[f];
  const double area = g.w;
  double nrm[3] = {g.x, g.y, g.z};
  const double *pa = pos + 3 * (size_t)e.x;
  double dri[3] = {c.x - pa[0], c.y - pa[1], c.z - pa[2]};
  unsigned char code = 0;
  if (bnd[i] != NO_BOUNDARY) {
    i = e.y; j = e.x;
    nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
    dri[0] = -dri[0]; dri[1] = -dri[1]; dri[2] = -dri[2];
    code |= F_SWAP;
  }
  const int jb = bnd[j];
  if (jb != NO_BOUNDARY) code |= F_SKIPJ;
  const double dtI = t_global - tlast[i], dtJ = t_global - tlast[j];
  const double dt = smin(dtI, dtJ);
  const double dti = dtI - 0.5 * dt, dtj = dtJ - 0.5 * dt;
  const double dsh = dri[0] * nrm[0] + dri[1] * nrm[1] + dri[2] * nrm[2];
  const double dsl = 2.0 * dsh;
  const double drj[3] = {dri[0] - nrm[0] * dsl, dri[1] - nrm[1] * dsl, dri[2] - nrm[2] * dsl};
  const double *ri = Wrec + 50 * (size_t)i, *rj = Wrec + 50 * (size_t)j;
  double Wi[NF], Wj[NF];
  if (jb != NO_BOUNDARY) {
#pragma unroll
    for (int k = 0; k < NF; k++) Wi[k] = Wj[k] = ri[k];
  } else {
    const double *ti = tau + 10 * (size_t)i, *tj = tau + 10 * (size_t)j;
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const double a = ti[k], b = tj[k];
      Wi[k] = ri[k] + (((ri[10 + k] * a) * dri[0] + (ri[20 + k] * a) * dri[1] + (ri[30 + k] * a) * dri[2]) +
                       (ri[40 + k] * a) * dti);
      Wj[k] = rj[k] + (((rj[10 + k] * b) * drj[0] + (rj[20 + k] * b) * drj[1] + (rj[30 + k] * b) * drj[2]) +
                       (rj[40 + k] * b) * dtj);
    }
  }
  const double *vi = vel + 3 * (size_t)i, *vj = vel + 3 * (size_t)j;
  const double fij[3] = {dri[0] - nrm[0] * dsh, dri[1] - nrm[1] * dsh, dri[2] - nrm[2] * dsh};
  const double fdv = (vj[0] - vi[0]) * fij[0] + (vj[1] - vi[1]) * fij[1] + (vj[2] - vi[2]) * fij[2];
  const double ids2 = -0.5 * fdv * ((dsh > 0.0) ? 1.0 / sqr(dsh) : 0.0);
  const double wij[3] = {(vj[0] + vi[0]) * 0.5 + dri[0] * ids2, (vj[1] + vi[1]) * 0.5 + dri[1] * ids2,
                         (vj[2] + vi[2]) * 0.5 + dri[2] * ids2};
  double psi, Bn, flux[NF];
  compute_flux<double>(P, wij, Wi, Wj, jb, nrm, psi, Bn, flux);
  const double tarea = dt * area;
  double *o = fcon + 14 * (size_t)f;
#pragma unroll
  for (int k = 0; k < NF; k++) o[k] = flux[k] * tarea;
  const double pt = psi * tarea;
  o[10] = nrm[0] * pt; o[11] = nrm[1] * pt; o[12] = nrm[2] * pt;
  o[13] = Bn * tarea;
  fcode[f] = code;
}

// ---- compute_update cell pass (MPI/compute_update.cpp:274-498) -----------
__global__ void __launch_bounds__(128) k_corr_cell(int n, Params P, double t_global,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ s12,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ tlast, double *__restrict__ volp,
    const double *__restrict__ Wrec, const double *__restrict__ tau,
    const double *__restrict__ fcon, const unsigned char *__restrict__ fcode,
    double *__restrict__ U, double *__restrict__ dU, double *__restrict__ stepdU,
    unsigned long long *__restrict__ counters) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const unsigned char ac = act[c];
  if (!(ac & (A_ACTIVE | A_LNGB))) return;
  double s[14];
#pragma unroll
  for (int k = 0; k < 14; k++) s[k] = 0.0;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int f = lnk[q];
    const unsigned char code = fcode[f];
    if (code & F_OFF) continue;
    const int2 e = s12[f];
    const int fi = (code & F_SWAP) ? e.y : e.x;
    const double *o = fcon + 14 * (size_t)f;
    if (c == fi) {
#pragma unroll
      for (int k = 0; k < NF; k++) s[k] -= o[k];
      s[10] = s[10] + o[10]; s[11] = s[11] + o[11]; s[12] = s[12] + o[12];
      s[13] += o[13];
    } else {
      if (code & F_SKIPJ) continue;
#pragma unroll
      for (int k = 0; k < NF; k++) s[k] += o[k];
      s[10] = s[10] - o[10]; s[11] = s[11] - o[11]; s[12] = s[12] - o[12];
      s[13] -= o[13];
    }
  }
  double *d0 = dU + 14 * (size_t)c;
  if (!(ac & A_ACTIVE)) {
    // inactive neighbour: accumulate until its own step (collect_results,
    // MPI/distribute_work.cpp:714-720)
    if (stepdU) {
#pragma unroll
      for (int k = 0; k < 14; k++) stepdU[14 * (size_t)c + k] = s[k];
    }
    if (bnd[c] == NO_BOUNDARY) {
#pragma unroll
      for (int k = 0; k < NF; k++) d0[k] += s[k];
      d0[13] += s[13];
      d0[10] = d0[10] + s[10]; d0[11] = d0[11] + s[11]; d0[12] = d0[12] + s[12];
    }
    return;
  }
  const double V = cvol[c];
  if (bnd[c] != NO_BOUNDARY) {
    volp[c] = V;
#pragma unroll
    for (int k = 0; k < 14; k++) d0[k] = 0.0;
    if (stepdU) {
#pragma unroll
      for (int k = 0; k < 14; k++) stepdU[14 * (size_t)c + k] = s[k];
    }
    return;
  }
  double Uc[NF];
  const double *Ui = U + 10 * (size_t)c;
#pragma unroll
  for (int k = 0; k < NF; k++) Uc[k] = Ui[k] + (d0[k] + s[k]);
  const double divB = d0[13] + s[13];
  const double dPsi[3] = {d0[10] + s[10], d0[11] + s[11], d0[12] + s[12]};
  const double dt = t_global - tlast[c];
#pragma unroll
  for (int k = 0; k < 14; k++) d0[k] = 0.0;  // dU_local = 0 (collect_results)
  if (stepdU) {
    double *sd = stepdU + 14 * (size_t)c;
#pragma unroll
    for (int k = 0; k < 13; k++) sd[k] = 0.0;
    sd[13] = dt > 0.0 ? divB / dt / V : divB;
  }
  const double *r = Wrec + 50 * (size_t)c;
  const double *tc = tau + 10 * (size_t)c;
  double W1[NF];
  if (Uc[MASS] <= 0.0) {
    // failed-mass fallback (MPI/compute_update.cpp:438-468)
    atomicAdd(&counters[0], 1ULL);
    double Ut[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) W1[k] = r[k] + (r[40 + k] * tc[k]) * dt;
    to_conservative(W1, volp[c], Ut);
    to_primitive(Ut, V, W1);
  } else {
    const double dth = 0.5 * dt;
    double Wh[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) Wh[k] = r[k] + (r[40 + k] * tc[k]) * dth;
    Uc[WBX] -= Wh[VELX] * divB;
    Uc[WBY] -= Wh[VELY] * divB;
    Uc[WBZ] -= Wh[VELZ] * divB;
    // Dedner divergence cleaning (MPI/compute_update.cpp:373-387, 403-405)
    const double pres = pressure(P, Wh);
    const double B2 = Wh[BX] * Wh[BX] + Wh[BY] * Wh[BY] + Wh[BZ] * Wh[BZ];
    const double dcs2 = P.gamma * pres + B2;
    const double ch_sig = sqrt(dcs2 / Wh[DENS]);
    Uc[WBX] -= dPsi[0];
    Uc[WBY] -= dPsi[1];
    Uc[WBZ] -= dPsi[2];
    Uc[MPSI] -= dcs2 * divB;
    const double l_min = pow(V / (4.0 * M_PI / 3.0), 1.0 / 3.0);
    Uc[MPSI] *= exp(-0.5 * ch_sig / l_min * dt);
    to_primitive(Uc, V, W1);
  }
  volp[c] = V;
  W1[ETHM] = ethm_update(P, W1, pos + 3 * (size_t)c);
  if (W1[ETHM] <= 0.0) {
    atomicAdd(&counters[1], 1ULL);
    W1[ETHM] = ethm_from_entropy(P, W1);
  } else {
    W1[ENTR] = entropy_from_ethm(P, W1);
  }
  double Un[NF];
  to_conservative(W1, V, Un);
  double *Uo = U + 10 * (size_t)c;
#pragma unroll
  for (int k = 0; k < NF; k++) Uo[k] = Un[k];
}

// ---- compute_pvel (MPI/compute_pvel.cpp:5-52) -----------------------------
__global__ void k_pvel(int n, Params P, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
                       const double *__restrict__ U, const double *__restrict__ volp,
                       const double *__restrict__ cvol, const double *__restrict__ ccen,
                       const double *__restrict__ pos, double *__restrict__ vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(act[i] & A_ACTIVE)) return;
  double W[NF];
  to_primitive(U + 10 * (size_t)i, volp[i], W);
  double v[3] = {W[VELX], W[VELY], W[VELZ]};
  const double B2 = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
  const double cs2 = (P.gamma * pressure(P, W) + B2) / W[DENS];
  const double vel2 = W[VELX] * W[VELX] + W[VELY] * W[VELY] + W[VELZ] * W[VELZ];
  const double vabs = sqrt(cs2 + vel2);
  const double *cc = ccen + 3 * (size_t)i, *x = pos + 3 * (size_t)i;
  const double d3[3] = {cc[0] - x[0], cc[1] - x[1], cc[2] - x[2]};
  const double d = sqrt(d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2]);
  if (d != 0.0) {
    const double eta = 0.25f, ki = 1.0f, f1 = 0.9f, f2 = 1.1f;
    const double R = pow(cvol[i] * (3.0 / (4.0 * M_PI)), 1.0 / 3.0);
    const double fac = d / (eta * R);
    double f;
    if (fac < f1) f = 0.0;
    else if (fac < f2) f = (d - f1 * eta * R) / ((f2 - f1) * eta * R);
    else f = 1.0;
    const double tau = d / vabs;
    f *= ki / tau;
    v[0] += d3[0] * f; v[1] += d3[1] * f; v[2] += d3[2] * f;
    if (bnd[i] != NO_BOUNDARY) v[0] = v[1] = v[2] = 0.0;
  }
  double *vo = vel + 3 * (size_t)i;
  vo[0] = v[0]; vo[1] = v[1]; vo[2] = v[2];
}

// ---- compute_timestep(i) (MPI/compute_timestep.cpp:6-51) ------------------
__device__ double cell_timestep(const Params &P, int i, bool with_faces, const int *off, const int *lnk,
                                const int2 *s12, const int *bnd, const double *U, const double *volp,
                                const double *vel) {
  double W[NF];
  to_primitive(U + 10 * (size_t)i, volp[i], W);
  const double *pv = vel + 3 * (size_t)i;
  double csi = 0.0, vrel = 0.0;
  const bool b = bnd[i] != NO_BOUNDARY;
  if (!b) {
    const double Pi = pressure(P, W) * P.gamma;
    const double B2i = W[BX] * W[BX] + W[BY] * W[BY] + W[BZ] * W[BZ];
    csi = sqrt((Pi + B2i) / W[DENS]);
    const double s = with_faces ? 1.0 : 0.0;
    const double d[3] = {W[VELX] - pv[0] * s, W[VELY] - pv[1] * s, W[VELZ] - pv[2] * s};
    vrel = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  }
  const double h = pow(volp[i] / (4.0 * M_PI / 3.0), 1.0 / 3.0);
  double dti = h / (csi + vrel + 1.0 / FVM_HUGE);
  if (with_faces) {
    const double fac = b ? 0.0 : 1.0;
    for (int q = off[i]; q < off[i + 1]; q++) {
      const int2 e = s12[lnk[q]];
      const int j = e.x == i ? e.y : e.x;
      const double *vj = vel + 3 * (size_t)j;
      const double w3[3] = {(vj[0] + pv[0]) * 0.5, (vj[1] + pv[1]) * 0.5, (vj[2] + pv[2]) * 0.5};
      const double dw[3] = {vj[0] - pv[0], vj[1] - pv[1], vj[2] - pv[2]};
      const double r[3] = {W[VELX] - w3[0], W[VELY] - w3[1], W[VELZ] - w3[2]};
      const double rv = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const double dwa = sqrt(dw[0] * dw[0] + dw[1] * dw[1] + dw[2] * dw[2]);
      dti = smin(dti, h / smax(fac * (csi + rv), 1.0 / FVM_HUGE + dwa));
    }
  }
  return dti * P.courant;
}

__device__ __forceinline__ double extra_timestep(const Params &P, int i, const int *bnd, const double *pos,
                                                 const double *vel) {
  if (P.eos == 0 || bnd[i] != NO_BOUNDARY) return FVM_HUGE;
  const double *x = pos + 3 * (size_t)i, *v = vel + 3 * (size_t)i;
  const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  return P.courant * r / (1.0 / FVM_HUGE + sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
}

__device__ __forceinline__ void atomic_min_pos(double *addr, double v) {
  atomicMin((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// compute_timesteps(false) first loops (MPI/compute_timestep.cpp:78-96); the
// global minimum is reduced per warp before one atomic per warp
__global__ void k_timestep(int n, Params P, const int *__restrict__ off, const int *__restrict__ lnk,
                           const int2 *__restrict__ s12, const unsigned char *__restrict__ act,
                           const int *__restrict__ bnd, const double *__restrict__ U,
                           const double *__restrict__ volp, const double *__restrict__ vel,
                           const double *__restrict__ pos, const double *__restrict__ tlast,
                           const double *__restrict__ tend, double *__restrict__ dtl,
                           double *__restrict__ dmin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double vmin = FVM_HUGE;
  if (i < n) {
    const unsigned char a = act[i];
    if (!(a & (A_ACTIVE | A_LNGB))) {
      dtl[i] = FVM_HUGE;
    } else if (!(a & A_ACTIVE)) {
      dtl[i] = (tend[i] - tlast[i]) * (bnd[i] != NO_BOUNDARY ? -1.0 : 1.0);
    } else {
      const double dti = smin(extra_timestep(P, i, bnd, pos, vel),
                              cell_timestep(P, i, true, off, lnk, s12, bnd, U, volp, vel));
      vmin = dti;
      dtl[i] = bnd[i] != NO_BOUNDARY ? -1.0 * dti : dti;
    }
  }
  for (int o = 16; o > 0; o >>= 1) vmin = smin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0 && vmin < FVM_HUGE) atomic_min_pos(dmin, vmin);
}

// dt >= 8 dt_min halving (MPI/compute_timestep.cpp:103-104)
__global__ void k_halve(int n, const unsigned char *__restrict__ act, const double *__restrict__ dmin,
                        double *__restrict__ dtl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(act[i] & A_ACTIVE)) return;
  if (dtl[i] >= 8.0 * dmin[0]) dtl[i] *= 0.5;
}

// adjust_timesteps relaxation (MPI/compute_timestep.cpp:123-142).  The
// reference relaxes neighbour pairs sequentially in site order and the
// result depends on that order, so it is reproduced by one thread.
__global__ void k_adjust_seq(int n, const int *__restrict__ off, const int *__restrict__ lnk,
                             const int2 *__restrict__ s12, const unsigned char *__restrict__ act,
                             const int *__restrict__ bnd, double *__restrict__ dtl,
                             unsigned char *__restrict__ hash) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int i = 0; i < n; i++) {
    if (!(act[i] & A_ACTIVE) || bnd[i] != NO_BOUNDARY) continue;
    double di = dtl[i];
    for (int q = off[i]; q < off[i + 1]; q++) {
      const int2 e = s12[lnk[q]];
      const int j = e.x == i ? e.y : e.x;
      double dj = dtl[j];
      if (dj < 0.0) continue;
      hash[j] = 1;
      di = smin(di, 2.0 * dj);
      dj = smin(dj, 2.0 * di);
      dtl[j] = dj;
      dtl[i] = di;
    }
  }
}

// rung assignment and inactive-neighbour promotion (MPI/compute_timestep.cpp
// :144-199) fused with collect_results (MPI/distribute_work.cpp:676-713) and
// the tlast/tend update of correct() (set_problem.cpp generic hook)
__global__ void k_rungs(int n, Params P, double t_global, int min_rung, int shared,
                        const unsigned char *__restrict__ act, const unsigned char *__restrict__ hash,
                        const double *__restrict__ dtl, const double *__restrict__ dmin,
                        int *__restrict__ rung, double *__restrict__ tlast, double *__restrict__ tend,
                        double *__restrict__ Wrec, int *__restrict__ iscal) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned char a = act[i];
  if (!(a & (A_ACTIVE | A_LNGB))) return;
  if (a & A_ACTIVE) {
    const int r = shared ? get_rung(P, dmin[0], min_rung) : get_rung(P, fabs(dtl[i]), min_rung);
    rung[i] = r;
    tlast[i] = t_global;
    tend[i] = t_global + get_dt(P, r);
    if (r < 0 || r >= RUNGMAX) atomicOr(&iscal[2], 1);
    return;
  }
  if (shared || !hash[i]) return;
  const double tl = tlast[i], te = tend[i];
  if (tl == t_global) return;
  if (!(te - tl > dtl[i])) return;
  const int rr = smax(exp_of(P.dtmax) - exp_of(fabs(0.5 * dtl[i])), 0);
  const double dt = get_dt(P, rr);
  int rn;
  double tn;
  if (tl + dt <= t_global) {
    rn = get_rung(P, dt, min_rung);
    tn = t_global + get_dt(P, rn);
    rn = -1 - rn;
  } else {
    rn = rr;
    tn = tl + dt;
  }
  if (tn - tl < te - tl) {
    rung[i] = rn < 0 ? -1 - rn : rn;
    tend[i] = tn;
    if (rn < 0) {
      double *w = Wrec + 50 * (size_t)i;
      for (int k = 10; k < 50; k++) w[k] = 0.0;
    }
  }
}

// distribute_fluid_update_data: primitives of the updated state
template <typename T>
__global__ void k_wst(int n, const unsigned char *__restrict__ act, const double *__restrict__ U,
                      const double *__restrict__ volp, T *__restrict__ Wst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(act[i] & (A_ACTIVE | A_LNGB))) return;
  double W[NF];
  to_primitive(U + 10 * (size_t)i, volp[i], W);
#pragma unroll
  for (int k = 0; k < NF; k++) Wst[10 * (size_t)i + k] = (T)W[k];
}

// ---- compute_update0 face pass (MPI/compute_update.cpp:713-810) ----------
__global__ void __launch_bounds__(128) k_pred_flux(int nf, Params P,
    const int2 *__restrict__ s12, const double4 *__restrict__ geo, const double4 *__restrict__ cen,
    const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ vel, const double *__restrict__ Wst,
    double *__restrict__ fcon, unsigned char *__restrict__ fcode) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int2 e = s12[f];
  if (!face_active(act, bnd, e.x, e.y)) { fcode[f] = F_OFF; return; }
  int i = e.x, j = e.y;
  const double4 g = geo[f], c = cen[f];
  const double area = g.w;
  double nrm[3] = {g.x, g.y, g.z};
  const double *pa = pos + 3 * (size_t)e.x;
  double dri[3] = {c.x - pa[0], c.y - pa[1], c.z - pa[2]};
  unsigned char code = 0;
  if (bnd[i] != NO_BOUNDARY) {
    i = e.y; j = e.x;
    nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2];
    dri[0] = -dri[0]; dri[1] = -dri[1]; dri[2] = -dri[2];
    code |= F_SWAP;
  }
  if (bnd[i] != NO_BOUNDARY) { fcode[f] = F_OFF; return; }
  const int jb = bnd[j];
  const double dsh = dri[0] * nrm[0] + dri[1] * nrm[1] + dri[2] * nrm[2];
  double Wi[NF], Wj[NF];
  const double *wi = Wst + 10 * (size_t)i, *wj = Wst + 10 * (size_t)(jb == NO_BOUNDARY ? j : i);
#pragma unroll
  for (int k = 0; k < NF; k++) { Wi[k] = wi[k]; Wj[k] = wj[k]; }
  const double *vi = vel + 3 * (size_t)i, *vj = vel + 3 * (size_t)j;
  const double fij[3] = {dri[0] - nrm[0] * dsh, dri[1] - nrm[1] * dsh, dri[2] - nrm[2] * dsh};
  const double fdv = (vj[0] - vi[0]) * fij[0] + (vj[1] - vi[1]) * fij[1] + (vj[2] - vi[2]) * fij[2];
  const double ids2 = -0.5 * fdv * ((dsh > 0.0) ? 1.0 / sqr(dsh) : 0.0);
  const double wij[3] = {(vj[0] + vi[0]) * 0.5 + dri[0] * ids2, (vj[1] + vi[1]) * 0.5 + dri[1] * ids2,
                         (vj[2] + vi[2]) * 0.5 + dri[2] * ids2};
  double psi, Bn, flux[NF];
  compute_flux<double>(P, wij, Wi, Wj, jb, nrm, psi, Bn, flux);
  double *o = fcon + 14 * (size_t)f;
#pragma unroll
  for (int k = 0; k < NF; k++) o[k] = flux[k] * area;
  const double pa2 = psi * area;
  o[10] = nrm[0] * pa2; o[11] = nrm[1] * pa2; o[12] = nrm[2] * pa2;
  o[13] = Bn * area;
  fcode[f] = code;
}

// ---- compute_update0 cell pass + collect_reconstruction -------------------
// (MPI/compute_update.cpp:812-964; MPI/distribute_work.cpp:820-834)
// Writes the predicted time derivative t into the cell's Wrec and the
// cell's final rung/tend.
__global__ void __launch_bounds__(128) k_pred_cell(int n, Params P, double t_global, int min_rung,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ s12,
    const double *__restrict__ cvol, const unsigned char *__restrict__ act, const int *__restrict__ bnd,
    const double *__restrict__ pos, const double *__restrict__ U,
    const double *__restrict__ fcon, const unsigned char *__restrict__ fcode,
    int *__restrict__ rung, double *__restrict__ tend, double *__restrict__ Wrec) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || !(act[c] & A_ACTIVE) || bnd[c] != NO_BOUNDARY) return;
  const double V = cvol[c];
  double dot[14];
#pragma unroll
  for (int k = 0; k < 14; k++) dot[k] = 0.0;
  for (int q = off[c]; q < off[c + 1]; q++) {
    const int f = lnk[q];
    const unsigned char code = fcode[f];
    if (code & F_OFF) continue;
    const int2 e = s12[f];
    const int fi = (code & F_SWAP) ? e.y : e.x;
    const double *o = fcon + 14 * (size_t)f;
    const double sg = c == fi ? -1.0 : 1.0;
#pragma unroll
    for (int k = 0; k < NF; k++) dot[k] = sg < 0.0 ? dot[k] - o[k] : dot[k] + o[k];
    dot[10] = sg < 0.0 ? dot[10] + o[10] : dot[10] - o[10];
    dot[11] = sg < 0.0 ? dot[11] + o[11] : dot[11] - o[11];
    dot[12] = sg < 0.0 ? dot[12] + o[12] : dot[12] - o[12];
    dot[13] = sg < 0.0 ? dot[13] + o[13] : dot[13] - o[13];
  }
  const double *U0 = U + 10 * (size_t)c;
  double u0[NF], W0[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) u0[k] = U0[k];
  to_primitive(u0, V, W0);
  int rg = rung[c];
  while (rg < RUNGMAX - 1 && u0[MASS] + dot[MASS] * get_dt(P, rg) <= 0.0 * u0[MASS]) rg++;
  const double dt = get_dt(P, rg);
  double Uc[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) Uc[k] = u0[k] + dot[k] * dt;
  {
    const double divB = dot[13];
    Uc[WBX] -= W0[VELX] * divB * dt;
    Uc[WBY] -= W0[VELY] * divB * dt;
    Uc[WBZ] -= W0[VELZ] * divB * dt;
    const double pres = pressure(P, W0);
    const double B2 = W0[BX] * W0[BX] + W0[BY] * W0[BY] + W0[BZ] * W0[BZ];
    const double dcs2 = P.gamma * pres + B2;
    const double ch_sig = sqrt(dcs2 / W0[DENS]);
    Uc[WBX] -= dot[10] * dt;
    Uc[WBY] -= dot[11] * dt;
    Uc[WBZ] -= dot[12] * dt;
    Uc[MPSI] -= dcs2 * divB * dt;
    const double l_min = pow(V / (4.0 * M_PI / 3.0), 1.0 / 3.0);
    Uc[MPSI] *= exp(-0.5 * ch_sig / l_min * dt);
  }
  double W1[NF];
  to_primitive(Uc, V, W1);
  W1[ETHM] = ethm_update(P, W1, pos + 3 * (size_t)c);
  if (W1[ETHM] <= 0.0) W1[ETHM] = W0[ETHM];
  else W1[ENTR] = entropy_from_ethm(P, W1);
  const double idt = 1.0 / dt;
  double *r = Wrec + 50 * (size_t)c;
#pragma unroll
  for (int k = 0; k < NF; k++) r[40 + k] = (W1[k] - W0[k]) * idt;
  // collect_reconstruction: rung = max(rung, get_rung(dt)), tend = t + dt(rung)
  int rf = rung[c];
  const int rb = get_rung(P, dt, min_rung);
  rf = rf < rb ? rb : rf;
  rung[c] = rf;
  tend[c] = t_global + get_dt(P, rf);
}

// ---- compute_reconstruction (MPI/compute_reconstruction.cpp:41-198) -------
// Two threads per active cell, five primitives each: Voronoi face gradient of
// the updated primitives, local limiter, density positivity rescale.
__global__ void __launch_bounds__(128) k_recon(int n, Params P,
    const int *__restrict__ off, const int *__restrict__ lnk, const int2 *__restrict__ s12,
    const double4 *__restrict__ geo, const double4 *__restrict__ cen, const double *__restrict__ cvol,
    const unsigned char *__restrict__ act, const int *__restrict__ bnd, const double *__restrict__ pos,
    const double *__restrict__ Wst, const int *__restrict__ rung, double *__restrict__ Wrec) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(t >> 1);
  const int k0 = (int)(t & 1) * KH;
  if (c >= n || !(act[c] & A_ACTIVE)) return;
  double *r = Wrec + 50 * (size_t)c + k0;
  const double *wsi = Wst + 10 * (size_t)c + k0;
  double Wi[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) Wi[k] = wsi[k];
  if (bnd[c] != NO_BOUNDARY) {
#pragma unroll
    for (int k = 0; k < KH; k++) { r[k] = Wi[k]; r[10 + k] = 0.0; r[20 + k] = 0.0; r[30 + k] = 0.0; r[40 + k] = 0.0; }
    return;
  }
  const int q0 = off[c], q1 = off[c + 1];
  double Wx[KH], Wy[KH], Wz[KH], mn[KH], mx[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { Wx[k] = Wy[k] = Wz[k] = mn[k] = mx[k] = 0.0; }
  const double *ip = pos + 3 * (size_t)c;
  const double px = ip[0], py = ip[1], pz = ip[2];
  double sc[3] = {0.0, 0.0, 0.0};
  bool zero = false;
  for (int q = q0; q < q1; q++) {
    const int f = lnk[q];
    const double4 g = geo[f], ce = cen[f];
    double d[3] = {ce.x - px, ce.y - py, ce.z - pz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double L = P.box[a];
      if (d[a] > 0.5 * L) d[a] -= L;
      else if (d[a] < -0.5 * L) d[a] += L;
    }
    sc[0] = sc[0] + d[0]; sc[1] = sc[1] + d[1]; sc[2] = sc[2] + d[2];
    const double area = g.w;
    const double sgn = (d[0] * g.x + d[1] * g.y + d[2] * g.z) < 0.0 ? -1.0 : 1.0;
    const double nrm[3] = {g.x * sgn, g.y * sgn, g.z * sgn};
    const double dsh = d[0] * nrm[0] + d[1] * nrm[1] + d[2] * nrm[2];
    const double idsA = area * ((dsh != 0.0) ? 0.5 / dsh : 0.0);
    const double drh[3] = {nrm[0] * dsh, nrm[1] * dsh, nrm[2] * dsh};
    const double fij[3] = {d[0] - drh[0], d[1] - drh[1], d[2] - drh[2]};
    const int2 e = s12[f];
    const int j = e.x == c ? e.y : e.x;
    if (bnd[j] != NO_BOUNDARY) { zero = true; break; }
    const double *Wj = Wst + 10 * (size_t)j + k0;
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const double wj = Wj[k];
      const double sum = wj + Wi[k];
      const double diff = wj - Wi[k];
      mn[k] = smin(mn[k], diff);
      mx[k] = smax(mx[k], diff);
      Wx[k] += (sum * drh[0] + diff * fij[0]) * idsA;
      Wy[k] += (sum * drh[1] + diff * fij[1]) * idsA;
      Wz[k] += (sum * drh[2] + diff * fij[2]) * idsA;
    }
  }
  if (zero) {
#pragma unroll
    for (int k = 0; k < KH; k++) { r[k] = Wi[k]; r[10 + k] = 0.0; r[20 + k] = 0.0; r[30 + k] = 0.0; r[40 + k] = 0.0; }
    return;
  }
  const double invV = 1.0 / cvol[c];
  double ln[KH], lq[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) { Wx[k] *= invV; Wy[k] *= invV; Wz[k] *= invV; ln[k] = 1.0; lq[k] = 1.0; }
  for (int q = q0; q < q1; q++) {
    const double4 ce = cen[lnk[q]];
    double d[3] = {ce.x - px, ce.y - py, ce.z - pz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double L = P.box[a];
      if (d[a] > 0.5 * L) d[a] -= L;
      else if (d[a] < -0.5 * L) d[a] += L;
    }
#pragma unroll
    for (int k = 0; k < KH; k++) {
      const double dWx = Wx[k] * d[0] + Wy[k] * d[1] + Wz[k] * d[2];
      limiter_min(ln[k], lq[k], dWx, mn[k], mx[k]);
    }
  }
  double tt[KH];
#pragma unroll
  for (int k = 0; k < KH; k++) {
    const double lm = ln[k] / lq[k];
    Wx[k] *= lm; Wy[k] *= lm; Wz[k] *= lm;
    tt[k] = r[40 + k] * lm;
  }
  if (k0 == 0) {  // density positivity for the *-state (MPI/compute_reconstruction.cpp:179-197)
    const double sum_dt = get_dt(P, rung[c]);
    const double dWx = Wx[0] * sc[0] + Wy[0] * sc[1] + Wz[0] * sc[2];
    const double dWp = dWx + tt[0] * sum_dt;
    const double dW = smax(dWx, dWp);
    if (dW > 0.0) {
      const double alpha = smin(1.0, 0.9 * Wi[0] / dW);
      Wx[0] *= alpha; Wy[0] *= alpha; Wz[0] *= alpha; tt[0] *= alpha;
    }
  }
#pragma unroll
  for (int k = 0; k < KH; k++) { r[k] = Wi[k]; r[10 + k] = Wx[k]; r[20 + k] = Wy[k]; r[30 + k] = Wz[k]; r[40 + k] = tt[k]; }
}

__global__ void k_shared_sync(int n, Params P, double t_global, const unsigned char *__restrict__ act,
                              const int *__restrict__ iscal, int *__restrict__ rung, double *__restrict__ tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(act[i] & A_ACTIVE)) return;
  const int r = iscal[0];
  rung[i] = r;
  tend[i] = t_global + get_dt(P, r);
}

__global__ void k_maxrung(int n, const int *__restrict__ rung, int *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int r = i < n ? rung[i] : 0;
  for (int o = 16; o > 0; o >>= 1) r = max(r, __shfl_xor_sync(0xffffffffu, r, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, r);
}

// ---- init: compute_pvel + compute_timesteps(true) -------------------------
__global__ void k_init_dt(int n, Params P, const int *__restrict__ bnd, const double *__restrict__ U,
                          const double *__restrict__ volp, const double *__restrict__ vel,
                          const double *__restrict__ pos, double *__restrict__ dmin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double vmin = FVM_HUGE;
  if (i < n)
    vmin = smin(extra_timestep(P, i, bnd, pos, vel),
                cell_timestep(P, i, false, nullptr, nullptr, nullptr, bnd, U, volp, vel));
  for (int o = 16; o > 0; o >>= 1) vmin = smin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
  if ((threadIdx.x & 31) == 0) atomic_min_pos(dmin, vmin);
}

__global__ void k_init_state(int n, const double *__restrict__ W, const double *__restrict__ cvol,
                             double *__restrict__ U, double *__restrict__ dU, double *__restrict__ Wrec,
                             double *__restrict__ volp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double w[NF], u[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) w[k] = W[10 * (size_t)i + k];
  to_conservative(w, cvol[i], u);
#pragma unroll
  for (int k = 0; k < NF; k++) U[10 * (size_t)i + k] = u[k];
  for (int k = 0; k < 14; k++) dU[14 * (size_t)i + k] = 0.0;
  for (int k = 0; k < 50; k++) Wrec[50 * (size_t)i + k] = k < NF ? w[k] : 0.0;
  volp[i] = cvol[i];
}

__global__ void k_limited_wrec(int n, const unsigned char *__restrict__ act, const double *__restrict__ Wrec,
                               const double *__restrict__ tau, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *r = Wrec + 50 * (size_t)i;
  double *o = out + 50 * (size_t)i;
  const bool imp = act[i] & (A_ACTIVE | A_LNGB);
  for (int k = 0; k < 50; k++) {
    const int v = k % 10;
    o[k] = (k >= 10 && imp) ? r[k] * tau[10 * (size_t)i + v] : r[k];
  }
}

__global__ void k_flux_kat(int nf, Params P, const double *wij, const double *Wi, const double *Wj,
                           const int *jbnd, const double *nrm, double *psi, double *Bn, double *flux) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double a[NF], b[NF], F[NF], w[3], nn[3], p, bn;
  for (int k = 0; k < NF; k++) { a[k] = Wi[10 * (size_t)f + k]; b[k] = Wj[10 * (size_t)f + k]; }
  for (int k = 0; k < 3; k++) { w[k] = wij[3 * (size_t)f + k]; nn[k] = nrm[3 * (size_t)f + k]; }
  compute_flux<double>(P, w, a, b, jbnd ? jbnd[f] : 0, nn, p, bn, F);
  psi[f] = p;
  Bn[f] = bn;
  for (int k = 0; k < NF; k++) flux[10 * (size_t)f + k] = F[k];
}

inline int nblk(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

// ============================== host context ================================

enum KernelId { KT_FLAGS = 0, KT_LIMITER, KT_CORR_FLUX, KT_CORR_CELL, KT_PVEL, KT_TIMESTEP, KT_RUNGS,
                KT_WST, KT_PRED_FLUX, KT_PRED_CELL, KT_RECON, KT_SYNC, KT_COUNT };
static const char *kKernelNames[KT_COUNT] = {"flags", "limiter", "corr_flux", "corr_cell", "pvel", "timestep",
                                             "rungs", "wst", "pred_flux", "pred_cell", "recon", "sync"};

struct fvm_ctx {
  int device;
  // per-kernel CUDA-event timing (enabled by fvm_set_profiling)
  bool prof;
  cudaEvent_t kev[2 * KT_COUNT];
  bool kev_pending[KT_COUNT];
  double kt_ms[KT_COUNT];
  long long kt_calls[KT_COUNT];
  long long launches;
  cudaStream_t st;
  cudaEvent_t ev0, ev1;
  fvm_params prm;
  Params P;
  int n, nf;
  long long nl;
  // scheduler (MPI/Scheduler.h)
  unsigned long long tsysU;
  int min_rung, max_rung;
  double t_global;
  bool have_mesh, have_state, in_step;
  unsigned long long cur_flags;
  Dev d;
  std::vector<long long> h_off;
  std::vector<int> h_ids;
  bool keep_step_dU;
  float last_ms;
  std::string err;
};

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      c->err = std::string(#call) + ": " + cudaGetErrorString(e_);                        \
      return FVM_ECUDA;                                                                   \
    }                                                                                     \
  } while (0)

#define LAUNCH_CHECK()                                                                    \
  do {                                                                                    \
    c->launches++;                                                                        \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      c->err = std::string("kernel launch: ") + cudaGetErrorString(e_);                   \
      return FVM_ECUDA;                                                                   \
    }                                                                                     \
  } while (0)

static void kt_begin(fvm_ctx *c, int id) {
  if (c->prof) cudaEventRecord(c->kev[2 * id], c->st);
}
static void kt_end(fvm_ctx *c, int id) {
  if (c->prof) {
    cudaEventRecord(c->kev[2 * id + 1], c->st);
    c->kev_pending[id] = true;
  }
}
// called after a stream synchronisation: fold pending event pairs into totals
static void kt_collect(fvm_ctx *c) {
  if (!c->prof) return;
  for (int k = 0; k < KT_COUNT; k++)
    if (c->kev_pending[k]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->kev[2 * k], c->kev[2 * k + 1]) == cudaSuccess) {
        c->kt_ms[k] += ms;
        c->kt_calls[k]++;
      }
      c->kev_pending[k] = false;
    }
}

template <typename T>
static int dalloc(fvm_ctx *c, T **p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
  if (e != cudaSuccess) {
    c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return FVM_ENOMEM;
  }
  return 0;
}

static void free_all(fvm_ctx *c) {
  void **ptrs = (void **)&c->d;
  for (size_t k = 0; k < sizeof(Dev) / sizeof(void *); k++)
    if (ptrs[k]) cudaFree(ptrs[k]);
  memset(&c->d, 0, sizeof(Dev));
}

extern "C" {

fvm_ctx *fvm_create(const fvm_params *p, int device) {
  if (!p) return nullptr;
  fvm_ctx *c = new fvm_ctx();
  c->device = device;
  c->prm = *p;
  memset(&c->d, 0, sizeof(Dev));
  c->P.gamma = p->gamma;
  c->P.courant = p->courant;
  for (int a = 0; a < 3; a++) c->P.box[a] = p->box[a];
  c->P.dtmax = p->dtmax;
  c->P.dt_tick = p->dtmax / (double)(1ULL << (RUNGMAX - 1));
  c->P.eos = p->eos;
  c->P.iso_GM = p->iso_GM;
  c->P.iso_cfac = p->iso_cfac;
  c->tsysU = 0;
  c->min_rung = 0;
  c->max_rung = RUNGMAX - 1;
  c->t_global = 0.0;
  c->keep_step_dU = getenv("FVM_KEEP_STEP_DU") != nullptr;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return nullptr;
  }
  for (int k = 0; k < 2 * KT_COUNT; k++) cudaEventCreate(&c->kev[k]);
  return c;
}

void fvm_destroy(fvm_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  free_all(c);
  for (int k = 0; k < 2 * KT_COUNT; k++) cudaEventDestroy(c->kev[k]);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaStreamDestroy(c->st);
  delete c;
}

const char *fvm_last_error(const fvm_ctx *c) { return c ? c->err.c_str() : "null context"; }

int fvm_set_mesh(fvm_ctx *c, int ncell, int nface, const int *s1, const int *s2, const double *n,
                 const double *centroid, const double *cell_volume, const double *cell_centroid,
                 const long long *off, const int *ids) {
  if (!c || ncell <= 0 || nface < 0 || !s1 || !s2 || !n || !centroid || !cell_volume || !cell_centroid || !off || !ids) {
    if (c) c->err = "fvm_set_mesh: bad argument";
    return FVM_EINVAL;
  }
  const long long nl = off[ncell];
  if (off[0] != 0 || nl < 0 || nl > 0x7fffffffLL) { c->err = "fvm_set_mesh: bad CSR offsets"; return FVM_EINVAL; }
  for (int f = 0; f < nface; f++)
    if (s1[f] < 0 || s1[f] >= ncell || s2[f] < 0 || s2[f] >= ncell || s1[f] == s2[f]) {
      c->err = "fvm_set_mesh: face " + std::to_string(f) + " has a bad cell index";
      return FVM_EINVAL;
    }
  for (long long q = 0; q < nl; q++)
    if (ids[q] < 0 || ids[q] >= nface) { c->err = "fvm_set_mesh: bad face id in cell lists"; return FVM_EINVAL; }
  for (int i = 0; i < ncell; i++)
    if (off[i + 1] < off[i]) { c->err = "fvm_set_mesh: CSR offsets decrease"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  free_all(c);
  c->n = ncell;
  c->nf = nface;
  c->nl = nl;
  int rc = 0;
  Dev &d = c->d;
  rc |= dalloc(c, &d.s12, nface); rc |= dalloc(c, &d.geo, nface); rc |= dalloc(c, &d.cen, nface);
  rc |= dalloc(c, &d.cvol, ncell); rc |= dalloc(c, &d.ccen, 3 * (size_t)ncell);
  rc |= dalloc(c, &d.off, ncell + 1); rc |= dalloc(c, &d.lnk, nl);
  rc |= dalloc(c, &d.pos, 3 * (size_t)ncell); rc |= dalloc(c, &d.vel, 3 * (size_t)ncell);
  rc |= dalloc(c, &d.tlast, ncell); rc |= dalloc(c, &d.tend, ncell); rc |= dalloc(c, &d.volp, ncell);
  rc |= dalloc(c, &d.rung, ncell); rc |= dalloc(c, &d.bnd, ncell);
  rc |= dalloc(c, &d.U, 10 * (size_t)ncell); rc |= dalloc(c, &d.dU, 14 * (size_t)ncell);
  rc |= dalloc(c, &d.Wrec, 50 * (size_t)ncell);
  rc |= dalloc(c, &d.act0, ncell); rc |= dalloc(c, &d.act, ncell); rc |= dalloc(c, &d.hash, ncell);
  rc |= dalloc(c, &d.fcode, nface); rc |= dalloc(c, &d.fcode2, nface);
  rc |= dalloc(c, &d.tau, 10 * (size_t)ncell); rc |= dalloc(c, &d.fcon, 14 * (size_t)nface);
  rc |= dalloc(c, &d.fcon2, 14 * (size_t)nface); rc |= dalloc(c, &d.Wst, 10 * (size_t)ncell);
  rc |= dalloc(c, &d.dtl, ncell);
  if (c->keep_step_dU) rc |= dalloc(c, &d.stepdU, 14 * (size_t)ncell);
  rc |= dalloc(c, &d.dscal, 4); rc |= dalloc(c, &d.iscal, 8); rc |= dalloc(c, &d.counters, 4);
  if (rc) return FVM_ENOMEM;
  std::vector<int2> hs(nface);
  std::vector<double4> hg(nface), hc(nface);
  for (int f = 0; f < nface; f++) {
    hs[f] = make_int2(s1[f], s2[f]);
    const double *v = n + 3 * (size_t)f;
    const double area = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double ia = 1.0 / area;
    hg[f] = make_double4(v[0] * ia, v[1] * ia, v[2] * ia, area);
    const double *q = centroid + 3 * (size_t)f;
    hc[f] = make_double4(q[0], q[1], q[2], 0.0);
  }
  std::vector<int> hoff(ncell + 1);
  for (int i = 0; i <= ncell; i++) hoff[i] = (int)off[i];
  c->h_off.assign(off, off + ncell + 1);
  c->h_ids.assign(ids, ids + nl);
  CK(cudaMemcpy(d.s12, hs.data(), sizeof(int2) * nface, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.geo, hg.data(), sizeof(double4) * nface, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.cen, hc.data(), sizeof(double4) * nface, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.cvol, cell_volume, sizeof(double) * ncell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.ccen, cell_centroid, sizeof(double) * 3 * ncell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.off, hoff.data(), sizeof(int) * (ncell + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.lnk, ids, sizeof(int) * nl, cudaMemcpyHostToDevice));
  CK(cudaMemsetAsync(d.counters, 0, 4 * sizeof(unsigned long long), c->st));
  CK(cudaStreamSynchronize(c->st));
  c->have_mesh = true;
  c->have_state = false;
  return 0;
}

static int sched_max_rung(fvm_ctx *c) {
  CK(cudaMemsetAsync(c->d.iscal, 0, sizeof(int), c->st));
  k_maxrung<<<nblk(c->n, 256), 256, 0, c->st>>>(c->n, c->d.rung, c->d.iscal);
  LAUNCH_CHECK();
  int r = 0;
  CK(cudaMemcpyAsync(&r, c->d.iscal, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->max_rung = r;
  return 0;
}

int fvm_init_problem(fvm_ctx *c, const double *W, const double *pos, const int *bnd, int rung_offset) {
  if (!c || !W || !pos) { if (c) c->err = "fvm_init_problem: bad argument"; return FVM_EINVAL; }
  if (!c->have_mesh) { c->err = "fvm_init_problem: no mesh"; return FVM_ENOMESH; }
  CK(cudaSetDevice(c->device));
  const int n = c->n;
  Dev &d = c->d;
  double *dW = nullptr;
  CK(cudaMalloc(&dW, sizeof(double) * 10 * (size_t)n));
  cudaError_t e = cudaMemcpyAsync(dW, W, sizeof(double) * 10 * (size_t)n, cudaMemcpyHostToDevice, c->st);
  if (e != cudaSuccess) { cudaFree(dW); c->err = cudaGetErrorString(e); return FVM_ECUDA; }
  CK(cudaMemcpyAsync(d.pos, pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, c->st));
  if (bnd) CK(cudaMemcpyAsync(d.bnd, bnd, sizeof(int) * n, cudaMemcpyHostToDevice, c->st));
  else CK(cudaMemsetAsync(d.bnd, 0, sizeof(int) * n, c->st));
  CK(cudaMemsetAsync(d.vel, 0, sizeof(double) * 3 * (size_t)n, c->st));
  CK(cudaMemsetAsync(d.tlast, 0, sizeof(double) * n, c->st));
  k_init_state<<<nblk(n, 128), 128, 0, c->st>>>(n, dW, d.cvol, d.U, d.dU, d.Wrec, d.volp);
  LAUNCH_CHECK();
  // compute_pvel on all cells, then the shared timestep
  CK(cudaMemsetAsync(d.act, A_ACTIVE, n, c->st));
  k_pvel<<<nblk(n, 128), 128, 0, c->st>>>(n, c->P, d.act, d.bnd, d.U, d.volp, d.cvol, d.ccen, d.pos, d.vel);
  LAUNCH_CHECK();
  const double hugev = FVM_HUGE;
  CK(cudaMemcpyAsync(d.dscal, &hugev, sizeof(double), cudaMemcpyHostToDevice, c->st));
  k_init_dt<<<nblk(n, 128), 128, 0, c->st>>>(n, c->P, d.bnd, d.U, d.volp, d.vel, d.pos, d.dscal);
  LAUNCH_CHECK();
  double dtmin = 0.0;
  CK(cudaMemcpyAsync(&dtmin, d.dscal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  cudaFree(dW);
  c->min_rung = 0;
  const int rung = get_rung(c->P, dtmin, c->min_rung) + rung_offset;
  if (rung < 0 || rung >= RUNGMAX - 1) { c->err = "fvm_init_problem: initial rung out of range"; return FVM_ERANGE; }
  std::vector<int> hr(n, rung);
  std::vector<double> ht(n, 0.0 + get_dt(c->P, rung));
  CK(cudaMemcpy(d.rung, hr.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.tend, ht.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  c->tsysU = 0;
  c->t_global = 0.0;
  c->max_rung = rung;
  c->have_state = true;
  c->in_step = false;
  return 0;
}

int fvm_get_state(fvm_ctx *c, double *pos, double *vel, double *tlast, double *tend, int *rung, double *U,
                  double *dU, double *wrec) {
  if (!c || !c->have_mesh) return FVM_ENOMESH;
  CK(cudaSetDevice(c->device));
  const size_t n = c->n;
  cudaStream_t s = c->st;
  if (pos) CK(cudaMemcpyAsync(pos, c->d.pos, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (vel) CK(cudaMemcpyAsync(vel, c->d.vel, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (tlast) CK(cudaMemcpyAsync(tlast, c->d.tlast, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (tend) CK(cudaMemcpyAsync(tend, c->d.tend, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (rung) CK(cudaMemcpyAsync(rung, c->d.rung, n * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (U) CK(cudaMemcpyAsync(U, c->d.U, 10 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (dU) CK(cudaMemcpyAsync(dU, c->d.dU, 14 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (wrec) CK(cudaMemcpyAsync(wrec, c->d.Wrec, 50 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int fvm_set_state(fvm_ctx *c, const double *vel, const double *tlast, const double *tend, const int *rung,
                  const double *U, const double *dU, const double *wrec, unsigned long long tsys_ticks) {
  if (!c || !c->have_mesh) return FVM_ENOMESH;
  if (c->in_step) { c->err = "fvm_set_state: inside a step"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const size_t n = c->n;
  cudaStream_t s = c->st;
  if (rung) {
    for (size_t i = 0; i < n; i++)
      if (rung[i] < 0 || rung[i] >= RUNGMAX - 1) { c->err = "fvm_set_state: rung out of range"; return FVM_ERANGE; }
    CK(cudaMemcpyAsync(c->d.rung, rung, n * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  if (vel) CK(cudaMemcpyAsync(c->d.vel, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (tlast) CK(cudaMemcpyAsync(c->d.tlast, tlast, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (tend) CK(cudaMemcpyAsync(c->d.tend, tend, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (U) CK(cudaMemcpyAsync(c->d.U, U, 10 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (dU) CK(cudaMemcpyAsync(c->d.dU, dU, 14 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (wrec) CK(cudaMemcpyAsync(c->d.Wrec, wrec, 50 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(c->d.volp, c->d.cvol, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  c->tsysU = tsys_ticks;
  c->t_global = c->P.dt_tick * (double)tsys_ticks;
  c->have_state = true;
  return sched_max_rung(c);
}

int fvm_begin_step(fvm_ctx *c) {
  if (!c || !c->have_state) { if (c) c->err = "fvm_begin_step: no state"; return FVM_ENOMESH; }
  if (c->in_step) { c->err = "fvm_begin_step: previous step not finished"; return FVM_EINVAL; }
  CK(cudaSetDevice(c->device));
  const int max_rung = c->max_rung;
  if (max_rung < 0 || max_rung >= RUNGMAX - 1) { c->err = "fvm_begin_step: max rung out of range"; return FVM_ERANGE; }
  // Scheduler::pull_active_list (MPI/Scheduler.h:108-154)
  const unsigned long long dtU = 1ULL << (RUNGMAX - 1 - max_rung);
  const unsigned long long tnextU = (c->tsysU / dtU + 1) * dtU;
  const unsigned long long flags = c->tsysU ^ tnextU;
  for (int b = 0; b < RUNGMAX; b++)
    if (flags & (1ULL << b)) c->min_rung = RUNGMAX - 1 - b;
  c->tsysU = tnextU;
  c->t_global = c->P.dt_tick * (double)c->tsysU;
  c->cur_flags = flags;
  const int n = c->n;
  Dev &d = c->d;
  CK(cudaMemsetAsync(d.iscal, 0, 8 * sizeof(int), c->st));
  kt_begin(c, KT_FLAGS);
  k_active<<<nblk(n, 256), 256, 0, c->st>>>(n, d.rung, flags, d.act0);
  LAUNCH_CHECK();
  k_ngbflags<<<nblk(n, 128), 128, 0, c->st>>>(n, d.off, d.lnk, d.s12, d.act0, d.act, d.iscal);
  LAUNCH_CHECK();
  kt_end(c, KT_FLAGS);
  c->in_step = true;
  return 0;
}

int fvm_slope_limiter(fvm_ctx *c) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_slope_limiter: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  kt_begin(c, KT_LIMITER);
  k_limiter<<<nblk(2LL * c->n, 128), 128, 0, c->st>>>(c->n, c->P, c->t_global, d.off, d.lnk, d.s12, d.geo, d.cen,
                                                 d.act, d.bnd, d.pos, d.tlast, d.Wrec, d.tau);
  LAUNCH_CHECK();
  kt_end(c, KT_LIMITER);
  return 0;
}

int fvm_compute_update(fvm_ctx *c) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_compute_update: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  kt_begin(c, KT_CORR_FLUX);
  k_corr_flux<<<nblk(c->nf, 128), 128, 0, c->st>>>(c->nf, c->P, c->t_global, d.s12, d.geo, d.cen, d.act, d.bnd,
                                                   d.pos, d.vel, d.tlast, d.Wrec, d.tau, d.fcon, d.fcode);
  LAUNCH_CHECK();
  kt_end(c, KT_CORR_FLUX);
  kt_begin(c, KT_CORR_CELL);
  k_corr_cell<<<nblk(c->n, 128), 128, 0, c->st>>>(c->n, c->P, c->t_global, d.off, d.lnk, d.s12, d.cvol, d.act,
                                                  d.bnd, d.pos, d.tlast, d.volp, d.Wrec, d.tau, d.fcon, d.fcode,
                                                  d.U, d.dU, d.stepdU, d.counters);
  LAUNCH_CHECK();
  kt_end(c, KT_CORR_CELL);
  return 0;
}

int fvm_compute_pvel(fvm_ctx *c) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_compute_pvel: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  kt_begin(c, KT_PVEL);
  k_pvel<<<nblk(c->n, 128), 128, 0, c->st>>>(c->n, c->P, d.act, d.bnd, d.U, d.volp, d.cvol, d.ccen, d.pos, d.vel);
  LAUNCH_CHECK();
  kt_end(c, KT_PVEL);
  return 0;
}

int fvm_compute_timesteps(fvm_ctx *c, int shared, double *dt_min_out) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_compute_timesteps: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  const int n = c->n;
  const double hugev = FVM_HUGE;
  CK(cudaMemcpyAsync(d.dscal, &hugev, sizeof(double), cudaMemcpyHostToDevice, c->st));
  kt_begin(c, KT_TIMESTEP);
  k_timestep<<<nblk(n, 128), 128, 0, c->st>>>(n, c->P, d.off, d.lnk, d.s12, d.act, d.bnd, d.U, d.volp, d.vel,
                                               d.pos, d.tlast, d.tend, d.dtl, d.dscal);
  LAUNCH_CHECK();
  kt_end(c, KT_TIMESTEP);
  if (!shared) {
    k_halve<<<nblk(n, 256), 256, 0, c->st>>>(n, d.act, d.dscal, d.dtl);
    LAUNCH_CHECK();
    CK(cudaMemsetAsync(d.hash, 0, n, c->st));
    k_adjust_seq<<<1, 32, 0, c->st>>>(n, d.off, d.lnk, d.s12, d.act, d.bnd, d.dtl, d.hash);
    LAUNCH_CHECK();
  }
  kt_begin(c, KT_RUNGS);
  k_rungs<<<nblk(n, 256), 256, 0, c->st>>>(n, c->P, c->t_global, c->min_rung, shared, d.act, d.hash, d.dtl,
                                            d.dscal, d.rung, d.tlast, d.tend, d.Wrec, d.iscal);
  LAUNCH_CHECK();
  kt_end(c, KT_RUNGS);
  if (dt_min_out) {
    CK(cudaMemcpyAsync(dt_min_out, d.dscal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return 0;
}

int fvm_collect_results(fvm_ctx *c) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_collect_results: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  kt_begin(c, KT_WST);
  k_wst<double><<<nblk(c->n, 256), 256, 0, c->st>>>(c->n, d.act, d.U, d.volp, d.Wst);
  LAUNCH_CHECK();
  kt_end(c, KT_WST);
  return 0;
}

int fvm_compute_update0(fvm_ctx *c) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_compute_update0: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  kt_begin(c, KT_PRED_FLUX);
  k_pred_flux<<<nblk(c->nf, 128), 128, 0, c->st>>>(c->nf, c->P, d.s12, d.geo, d.cen, d.act, d.bnd, d.pos, d.vel,
                                                   d.Wst, d.fcon2, d.fcode2);
  LAUNCH_CHECK();
  kt_end(c, KT_PRED_FLUX);
  return 0;
}

int fvm_compute_reconstruction(fvm_ctx *c) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_compute_reconstruction: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  kt_begin(c, KT_PRED_CELL);
  k_pred_cell<<<nblk(c->n, 128), 128, 0, c->st>>>(c->n, c->P, c->t_global, c->min_rung, d.off, d.lnk, d.s12,
                                                  d.cvol, d.act, d.bnd, d.pos, d.U, d.fcon2, d.fcode2, d.rung,
                                                  d.tend, d.Wrec);
  LAUNCH_CHECK();
  kt_end(c, KT_PRED_CELL);
  kt_begin(c, KT_RECON);
  k_recon<<<nblk(2LL * c->n, 128), 128, 0, c->st>>>(c->n, c->P, d.off, d.lnk, d.s12, d.geo, d.cen, d.cvol, d.act,
                                                    d.bnd, d.pos, d.Wst, d.rung, d.Wrec);
  LAUNCH_CHECK();
  kt_end(c, KT_RECON);
  return 0;
}

int fvm_end_step(fvm_ctx *c, int shared) {
  if (!c || !c->in_step) { if (c) c->err = "fvm_end_step: call fvm_begin_step first"; return FVM_EINVAL; }
  Dev &d = c->d;
  if (shared) {
    kt_begin(c, KT_SYNC);
  CK(cudaMemsetAsync(d.iscal, 0, sizeof(int), c->st));
  k_maxrung<<<nblk(c->n, 256), 256, 0, c->st>>>(c->n, d.rung, d.iscal);
  LAUNCH_CHECK();
  k_shared_sync<<<nblk(c->n, 256), 256, 0, c->st>>>(c->n, c->P, c->t_global, d.act, d.iscal, d.rung, d.tend);
    LAUNCH_CHECK();
  kt_end(c, KT_SYNC);
    int h[3];
    CK(cudaMemcpyAsync(h, d.iscal, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    kt_collect(c);
    c->in_step = false;
    if (h[2]) { c->err = "rung out of range"; return FVM_ERANGE; }
    c->max_rung = h[0];
    return h[1];
  }
  int h[3];
  CK(cudaMemcpyAsync(h, d.iscal, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  c->in_step = false;
  int rc = sched_max_rung(c);
  kt_collect(c);
  if (rc) return rc;
  if (h[2]) { c->err = "rung out of range"; return FVM_ERANGE; }
  return h[1];
}

int fvm_step(fvm_ctx *c, int shared) {
  int rc;
  if ((rc = fvm_begin_step(c)) < 0) return rc;
  CK(cudaEventRecord(c->ev0, c->st));
  if ((rc = fvm_slope_limiter(c)) < 0) return rc;
  if ((rc = fvm_compute_update(c)) < 0) return rc;
  if ((rc = fvm_compute_pvel(c)) < 0) return rc;
  if ((rc = fvm_compute_timesteps(c, shared, nullptr)) < 0) return rc;
  if ((rc = fvm_collect_results(c)) < 0) return rc;
  if ((rc = fvm_compute_update0(c)) < 0) return rc;
  if ((rc = fvm_compute_reconstruction(c)) < 0) return rc;
  CK(cudaEventRecord(c->ev1, c->st));
  rc = fvm_end_step(c, shared);
  cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
  return rc;
}

double fvm_time(const fvm_ctx *c) { return c ? c->t_global : 0.0; }

void *fvm_stream(fvm_ctx *c) { return c ? (void *)c->st : nullptr; }
long long fvm_launch_count(const fvm_ctx *c) { return c ? c->launches : 0; }

int fvm_set_profiling(fvm_ctx *c, int on) {
  if (!c) return FVM_EINVAL;
  c->prof = on != 0;
  for (int k = 0; k < KT_COUNT; k++) { c->kt_ms[k] = 0.0; c->kt_calls[k] = 0; c->kev_pending[k] = false; }
  return 0;
}

int fvm_kernel_times(const fvm_ctx *c, int k, const char **name, double *total_ms, long long *calls) {
  if (!c || k < 0) return FVM_EINVAL;
  if (k >= KT_COUNT) return 0;
  if (name) *name = kKernelNames[k];
  if (total_ms) *total_ms = c->kt_ms[k];
  if (calls) *calls = c->kt_calls[k];
  return 1;
}
unsigned long long fvm_tsys_ticks(const fvm_ctx *c) { return c ? c->tsysU : 0ULL; }
float fvm_last_step_ms(const fvm_ctx *c) { return c ? c->last_ms : 0.0f; }

int fvm_get_active_faces(fvm_ctx *c, int *ids, int *nout) {
  if (!c || !c->have_state) return FVM_ENOMESH;
  CK(cudaSetDevice(c->device));
  std::vector<unsigned char> act(c->n);
  std::vector<int> bnd(c->n);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(act.data(), c->d.act, c->n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(bnd.data(), c->d.bnd, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
  std::vector<unsigned char> seen(c->nf > 0 ? c->nf : 1, 0);
  int cnt = 0;
  for (int i = 0; i < c->n; i++) {
    if (!(act[i] & A_ACTIVE) || bnd[i] != NO_BOUNDARY) continue;
    for (long long q = c->h_off[i]; q < c->h_off[i + 1]; q++) {
      const int f = c->h_ids[q];
      if (seen[f]) continue;
      seen[f] = 1;
      if (ids) ids[cnt] = f;
      cnt++;
    }
  }
  if (nout) *nout = cnt;
  return 0;
}

int fvm_get_limited_wrec(fvm_ctx *c, double *wrec) {
  if (!c || !c->have_state || !wrec) return FVM_EINVAL;
  CK(cudaSetDevice(c->device));
  double *tmp = nullptr;
  CK(cudaMalloc(&tmp, 50 * sizeof(double) * (size_t)c->n));
  k_limited_wrec<<<nblk(c->n, 128), 128, 0, c->st>>>(c->n, c->d.act, c->d.Wrec, c->d.tau, tmp);
  cudaError_t e = cudaMemcpyAsync(wrec, tmp, 50 * sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->st);
  cudaStreamSynchronize(c->st);
  cudaFree(tmp);
  if (e != cudaSuccess) { c->err = cudaGetErrorString(e); return FVM_ECUDA; }
  return 0;
}

int fvm_get_step_dU(fvm_ctx *c, double *dU) {
  if (!c || !dU) return FVM_EINVAL;
  if (!c->d.stepdU) { c->err = "fvm_get_step_dU: set FVM_KEEP_STEP_DU before fvm_set_mesh"; return FVM_EINVAL; }
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(dU, c->d.stepdU, 14 * sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost));
  return 0;
}

int fvm_get_dt_list(fvm_ctx *c, double *dt) {
  if (!c || !dt || !c->have_mesh) return FVM_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(dt, c->d.dtl, sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost));
  return 0;
}

int fvm_get_counters(fvm_ctx *c, long long *out2) {
  if (!c || !out2 || !c->have_mesh) return FVM_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  unsigned long long h[2];
  CK(cudaMemcpy(h, c->d.counters, sizeof(h), cudaMemcpyDeviceToHost));
  out2[0] = (long long)h[0];
  out2[1] = (long long)h[1];
  return 0;
}

int fvm_compute_flux(fvm_ctx *c, int nface, const double *wij, const double *Wi, const double *Wj, const int *jbnd,
                     const double *normal, double *psi, double *Bn, double *flux) {
  if (!c || nface < 0 || !wij || !Wi || !Wj || !normal || !psi || !Bn || !flux) return FVM_EINVAL;
  if (nface == 0) return 0;
  CK(cudaSetDevice(c->device));
  const size_t nf = nface;
  const size_t bytes = sizeof(double) * nf * (3 + 10 + 10 + 3 + 1 + 1 + 10) + sizeof(int) * nf;
  char *buf = nullptr;
  CK(cudaMalloc(&buf, bytes));
  double *dw = (double *)buf, *da = dw + 3 * nf, *db = da + 10 * nf, *dn = db + 10 * nf, *dp = dn + 3 * nf,
         *dB = dp + nf, *dF = dB + nf;
  int *dj = (int *)(dF + 10 * nf);
  cudaMemcpyAsync(dw, wij, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(da, Wi, sizeof(double) * 10 * nf, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(db, Wj, sizeof(double) * 10 * nf, cudaMemcpyHostToDevice, c->st);
  cudaMemcpyAsync(dn, normal, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, c->st);
  if (jbnd) cudaMemcpyAsync(dj, jbnd, sizeof(int) * nf, cudaMemcpyHostToDevice, c->st);
  k_flux_kat<<<nblk(nface, 128), 128, 0, c->st>>>(nface, c->P, dw, da, db, jbnd ? dj : nullptr, dn, dp, dB, dF);
  cudaMemcpyAsync(psi, dp, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(Bn, dB, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(flux, dF, sizeof(double) * 10 * nf, cudaMemcpyDeviceToHost, c->st);
  cudaError_t e = cudaStreamSynchronize(c->st);
  cudaFree(buf);
  if (e != cudaSuccess) { c->err = cudaGetErrorString(e); return FVM_ECUDA; }
  return 0;
}

}  // extern "C"
