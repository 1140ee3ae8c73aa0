// Learned face flux inside the rotated-frame flux routine: the compute_flux
// hooks that gate a face, hand it to the network, harvest training pairs,
// and rebuild the flux from the network's output.
//
// The network does not replace the whole flux.  In the frame of the face
// (velocities shifted by the face speed w) the flux is split into the
// central part, the mean of the two sides' physical MHD fluxes, computed
// exactly, and the dissipative remainder of the HLLD solver.  To first order
// in the jump between the two sides that remainder is a matrix of the mean
// state times the jump, so it is written as m times a bounded function of
// the face: m is the size of the seven scaled jumps (density, three
// velocities, pressure, two tangential fields), and the network predicts the
// remainder divided by m from the side means, the jump's direction, m itself
// and the jump of the fast speed.  Its error is then relative to the
// dissipation on every face, however smooth, and m multiplies the output in
// FP32.  The HLLD solution is Galilean covariant under a normal boost (mass,
// momentum, energy and induction fluxes transform exactly), so the
// face-frame flux maps back to the moving face's flux without approximation.
//
// Included by fvm_kernels.cu after fvm_math.cuh and flux_mlp.cuh.
#pragma once

namespace fvm {

// Deferred-face buffers, harvest buffers and gate settings of one context.
// The gate: ideal-gas EOS, no boundary neighbour, small relative density and
// pressure jumps, bounded normal Mach number in the face frame, and every
// standardised network input within ZMAX spreads of its training mean.
struct LearnBuf {
  __half *X;  // [cap x 16] features of deferred faces (FP16, the network's input type)
  float *Y;          // [cap x 8] network outputs
  int *gface;        // [cap] face of each deferred slot
  int *count;        // deferred faces of the current pass
  float *hx, *hy;    // harvested (features, targets), [hcap x 16] and [hcap x 8]
  unsigned long long *hcount;
  long long hcap;
  unsigned hstride;  // harvest one gated face in hstride (hash-sampled)
  unsigned judge;    // judge one deferred face in `judge` against the exact solver (0: none)
  double *stats;     // see LSTAT_*
  const double *U;   // conserved state (positivity gate)
  const double *vol; // cell volumes (positivity gate: magnetic energy)
  const float *norm; // feature and output standardisation: mu_x[16], 1/sd_x[16], mu_y[8], sd_y[8]
  float drho, dp, mach;  // gate: relative density and pressure jumps, normal Mach number
  float jmax;            // gate: size m of the scaled jump (the network's x[14])
  int surrogate;     // dissipation of gated faces: SUR_NETWORK, SUR_CENTRAL (none) or SUR_LLF
};
enum { LSTAT_DEFERRED = 0, LSTAT_FALLBACK, LSTAT_JUDGED, LSTAT_ERR, LSTAT_REF, LSTAT_ERRMAX, LSTAT_POSFALL,
       LSTAT_COUNT = 8 };
// What stands in for the HLLD dissipation on gated faces.  The network is the
// product; the other two are the comparisons a test or benchmark runs on the
// same faces: the central flux alone (zero dissipation) and the local
// Lax-Friedrichs (Rusanov) dissipation.
enum { SUR_NETWORK = 0, SUR_CENTRAL = 1, SUR_LLF = 2 };

__device__ __forceinline__ unsigned face_hash(unsigned f, unsigned salt) {
  unsigned x = f * 0x9E3779B1u ^ (salt * 0x85EBCA77u + 0x165667B1u);
  x ^= x >> 15; x *= 0x2C1B3C6Du; x ^= x >> 12; x *= 0x297A2D39u; x ^= x >> 15;
  return x;
}

// Rotated-frame side states handed to the Riemann hook.
struct FaceSides {
  float Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR, BzR, chL, chR;
};

template <typename T>
__device__ __forceinline__ T flux_scale(int k, T rho, T c, T sr) {
  // MASS, MOMX..Z, ENER, WBX..Z
  return k == 0 ? rho * c : (k <= 3 ? rho * c * c : (k == 4 ? rho * c * c * c : sr * c * c));
}

// The seven scaled jumps of a face (density by the mean density, velocities
// by the larger fast speed c, pressure by rho c^2, tangential fields by
// sqrt(rho) c) and their size m, which the function returns.
__device__ __forceinline__ float scaled_jump(const FaceSides &s, float *j) {
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
  const float ic = 1.0f / c, iP = 1.0f / (rho * c * c), iB = 1.0f / (sr * c);
  j[0] = (s.dR - s.dL) / rho;
  j[1] = (s.vxR - s.vxL) * ic;
  j[2] = (s.vyR - s.vyL) * ic;
  j[3] = (s.vzR - s.vzL) * ic;
  j[4] = (s.pR - s.pL) * iP;
  j[5] = (s.ByR - s.ByL) * iB;
  j[6] = (s.BzR - s.BzL) * iB;
  float m2 = 0.0f;
#pragma unroll
  for (int k = 0; k < 7; k++) m2 = fmaf(j[k], j[k], m2);
  return sqrtf(m2);
}

// Features of a face (see the file comment): x[0..6] the side means of the
// normal velocity in the face frame, the tangential velocities, the pressure
// and the three field components; x[7..13] the direction of the scaled jump
// (density, velocities, pressure, tangential fields); x[14] its size m;
// x[15] the jump of the fast speed.  Velocities are scaled by the larger fast
// speed c, pressure by rho c^2 and fields by sqrt(rho) c, with rho the mean
// density.  Returns m.
__device__ __forceinline__ float face_features(const FaceSides &s, float *x) {
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
  const float ic = 1.0f / c, iP = 1.0f / (rho * c * c), iB = 1.0f / (sr * c);
  x[0] = (0.5f * (s.vxL + s.vxR) - s.w) * ic;
  x[1] = 0.5f * (s.vyL + s.vyR) * ic;
  x[2] = 0.5f * (s.vzL + s.vzR) * ic;
  x[3] = 0.5f * (s.pL + s.pR) * iP;
  x[4] = s.Bx * iB;
  x[5] = 0.5f * (s.ByL + s.ByR) * iB;
  x[6] = 0.5f * (s.BzL + s.BzR) * iB;
  float j[7];
  const float m = scaled_jump(s, j), im = m > 0.0f ? 1.0f / m : 0.0f;
#pragma unroll
  for (int k = 0; k < 7; k++) x[7 + k] = j[k] * im;
  x[14] = m;
  x[15] = (s.chR - s.chL) * ic;
  return m;
}

// Network inputs: the features standardised with the training set's mean and
// spread.  Returns false when one lies more than ZMAX spreads from the
// training mean (outside what the network has seen).
constexpr float ZMAX = 8.0f;
__device__ __forceinline__ bool net_inputs(const LearnBuf &lb, const FaceSides &s, float *x) {
  face_features(s, x);
  bool inside = true;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    x[k] = (x[k] - lb.norm[k]) * lb.norm[16 + k];
    inside = inside && fabsf(x[k]) <= ZMAX;
  }
  return inside;
}

// Mean of the two sides' physical fluxes in the face frame (u = vx - w).
template <typename T>
__device__ __forceinline__ void central_flux(const FaceSides &s, T *F) {
  T FL[8], FR[8];
  const float sides[2][8] = {{s.dL, s.pL, s.eL, s.vxL, s.vyL, s.vzL, s.ByL, s.BzL},
                             {s.dR, s.pR, s.eR, s.vxR, s.vyR, s.vzR, s.ByR, s.BzR}};
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const T d = sides[q][0], p = sides[q][1], e = sides[q][2], u = T(sides[q][3]) - T(s.w), v = sides[q][4],
            wz = sides[q][5], by = sides[q][6], bz = sides[q][7], bx = s.Bx;
    const T B2 = bx * bx + by * by + bz * bz;
    const T pT = p + T(0.5) * B2;
    const T et = e + T(0.5) * (d * (u * u + v * v + wz * wz) + B2);
    T *G = q ? FR : FL;
    G[0] = d * u;
    G[1] = d * u * u + pT - bx * bx;
    G[2] = d * v * u - bx * by;
    G[3] = d * wz * u - bx * bz;
    G[4] = (et + pT) * u - bx * (u * bx + v * by + wz * bz);
    G[5] = T(0);
    G[6] = by * u - bx * v;
    G[7] = bz * u - bx * wz;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) F[k] = T(0.5) * (FL[k] + FR[k]);
}

// The scaled dissipation of a face: the HLLD flux in the face frame minus the
// central flux, each output divided by its flux scale
// (MPI/compute_update.cpp:1109-1341 with w = 0).  T = double gives the
// training targets and the judge's reference: the side states are the
// solver's own (FP32 in the FP32 bulk path), and the double evaluation keeps
// the small difference free of cancellation error.
template <typename T>
__device__ __forceinline__ void face_targets(const FaceSides &s, T gamma, T *y) {
  T Fp[8], Fc[8];
  riemann_hlld<T>(gamma, Fp, T(s.Bx), T(0), T(s.dL), T(s.pL), T(s.eL), T(s.vxL) - T(s.w), T(s.vyL), T(s.vzL),
                  T(s.ByL), T(s.BzL), T(s.dR), T(s.pR), T(s.eR), T(s.vxR) - T(s.w), T(s.vyR), T(s.vzR), T(s.ByR),
                  T(s.BzR));
  central_flux<T>(s, Fc);
  const T rho = T(0.5) * (T(s.dL) + T(s.dR)), c = T(fmaxf(s.chL, s.chR)), sr = sqrt(rho);
#pragma unroll
  for (int k = 0; k < 8; k++) y[k] = (Fp[k] - Fc[k]) / flux_scale<T>(k, rho, c, sr);
}

// The local Lax-Friedrichs dissipation -S/2 (U_R - U_L) of the face-frame
// conserved state, S the larger of |u| + c_f on the two sides, in the scaled
// units of face_targets (the normal field's flux is not dissipated).
__device__ __forceinline__ void llf_outputs(const FaceSides &s, float *y) {
  const float uL = s.vxL - s.w, uR = s.vxR - s.w;
  const float S = fmaxf(fabsf(uL) + s.chL, fabsf(uR) + s.chR);
  const float B2L = s.Bx * s.Bx + s.ByL * s.ByL + s.BzL * s.BzL, B2R = s.Bx * s.Bx + s.ByR * s.ByR + s.BzR * s.BzR;
  const float EL = s.eL + 0.5f * (s.dL * (uL * uL + s.vyL * s.vyL + s.vzL * s.vzL) + B2L);
  const float ER = s.eR + 0.5f * (s.dR * (uR * uR + s.vyR * s.vyR + s.vzR * s.vzR) + B2R);
  const float dU[8] = {s.dR - s.dL, s.dR * uR - s.dL * uL, s.dR * s.vyR - s.dL * s.vyL, s.dR * s.vzR - s.dL * s.vzL,
                       ER - EL, 0.0f, s.ByR - s.ByL, s.BzR - s.BzL};
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
#pragma unroll
  for (int k = 0; k < 8; k++) y[k] = -0.5f * S * dU[k] / flux_scale<float>(k, rho, c, sr);
}

// Rotated lab-frame flux of the moving face from the (unstandardised)
// scaled dissipation y.
template <typename T>
__device__ __forceinline__ void flux_from_outputs(const FaceSides &s, const float *y, T *F) {
  float Fc[8];
  central_flux<float>(s, Fc);
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
  float Fp[8];
#pragma unroll
  for (int k = 0; k < 8; k++) Fp[k] = Fc[k] + y[k] * flux_scale<float>(k, rho, c, sr);
  const float w = s.w;
  F[MASS] = T(Fp[0]);
  F[MOMX] = T(Fp[1] + w * Fp[0]);
  F[MOMY] = T(Fp[2]);
  F[MOMZ] = T(Fp[3]);
  F[ENER] = T(Fp[4] + w * Fp[1] + 0.5f * w * w * Fp[0]);
  F[WBX] = T(-w * s.Bx);
  F[WBY] = T(Fp[6]);
  F[WBZ] = T(Fp[7]);
}

__device__ __forceinline__ bool face_gated(const Params &P, const LearnBuf &lb, const FaceSides &s, int jbnd) {
  if (P.eos != 0 || jbnd != NO_BOUNDARY) return false;
  const float rho = 0.5f * (s.dL + s.dR), pm = 0.5f * (s.pL + s.pR), c = fmaxf(s.chL, s.chR);
  const float un = 0.5f * (s.vxL + s.vxR) - s.w;
  if (!(fabsf(s.dR - s.dL) <= lb.drho * rho && fabsf(s.pR - s.pL) <= lb.dp * pm && fabsf(un) <= lb.mach * c &&
        s.dL > 0.0f && s.dR > 0.0f && s.pL > 0.0f && s.pR > 0.0f))
    return false;
  float j[7];
  return scaled_jump(s, j) <= lb.jmax;
}

template <typename T>
__device__ __forceinline__ FaceSides make_sides(T Bx, T w, T dens_L, T pres_L, T ethm_L, T velx_L, T vely_L,
                                                T velz_L, T By_L, T Bz_L, T dens_R, T pres_R, T ethm_R,
                                                T velx_R, T vely_R, T velz_R, T By_R, T Bz_R, T chL, T chR) {
  return FaceSides{float(Bx), float(w), float(dens_L), float(pres_L), float(ethm_L), float(velx_L),
                   float(vely_L), float(velz_L), float(By_L), float(Bz_L), float(dens_R), float(pres_R),
                   float(ethm_R), float(velx_R), float(vely_R), float(velz_R), float(By_R), float(Bz_R),
                   float(chL), float(chR)};
}

// Exact solve everywhere; gated faces sampled one in hstride also append
// their (features, targets) to the harvest buffers.
struct HarvestSolver {
  const Params &P;
  const LearnBuf &lb;
  unsigned f, salt;
  template <typename T>
  __device__ bool operator()(T gamma, T *F, T Bx, T w, T dL, T pL, T eL, T vxL, T vyL, T vzL, T ByL, T BzL, T dR,
                             T pR, T eR, T vxR, T vyR, T vzR, T ByR, T BzR, T chL, T chR, int jbnd) {
    riemann_hlld<T>(gamma, F, Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR, BzR);
    const FaceSides s = make_sides<T>(Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR,
                                      BzR, chL, chR);
    if (face_gated(P, lb, s, jbnd) && face_hash(f, salt) % lb.hstride == 0) {
      const unsigned long long slot = atomicAdd(lb.hcount, 1ull);
      if ((long long)slot < lb.hcap) {
        float x[16];
        double y[8];
        face_features(s, x);
        face_targets<double>(s, double(gamma), y);
#pragma unroll
        for (int k = 0; k < 16; k++) lb.hx[16 * slot + k] = x[k];
#pragma unroll
        for (int k = 0; k < 8; k++) lb.hy[8 * slot + k] = float(y[k]);
      }
    }
    return true;
  }
};

// Gated faces are deferred to the network (features written to their slot,
// false returned); the others are solved exactly.
struct DeferSolver {
  const Params &P;
  const LearnBuf &lb;
  int f;
  bool deferred = false;
  template <typename T>
  __device__ bool operator()(T gamma, T *F, T Bx, T w, T dL, T pL, T eL, T vxL, T vyL, T vzL, T ByL, T BzL, T dR,
                             T pR, T eR, T vxR, T vyR, T vzR, T ByR, T BzR, T chL, T chR, int jbnd) {
    const FaceSides s = make_sides<T>(Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR,
                                      BzR, chL, chR);
    float x[16];
    if (face_gated(P, lb, s, jbnd) && net_inputs(lb, s, x)) {
      const int slot = atomicAdd(lb.count, 1);
      uint4 *o = reinterpret_cast<uint4 *>(lb.X + 16 * (size_t)slot);
      o[0] = make_uint4(mlp::pack_f16(x[0], x[1]), mlp::pack_f16(x[2], x[3]), mlp::pack_f16(x[4], x[5]),
                        mlp::pack_f16(x[6], x[7]));
      o[1] = make_uint4(mlp::pack_f16(x[8], x[9]), mlp::pack_f16(x[10], x[11]), mlp::pack_f16(x[12], x[13]),
                        mlp::pack_f16(x[14], x[15]));
      lb.gface[slot] = f;
      deferred = true;
      return false;
    }
    riemann_hlld<T>(gamma, F, Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR, BzR);
    return true;
  }
};

// The flux of a deferred face from the network outputs y (scaled
// dissipation = m (mu_y + sd_y y)), or from the surrogate the context asks
// for; one slot in lb.judge is also solved exactly (in double) and the
// difference accumulated.
struct LearnedSolver {
  const LearnBuf &lb;
  float *y;  // network output, replaced by the scaled dissipation in place
  bool judged;
  template <typename T>
  __device__ bool operator()(T gamma, T *F, T Bx, T w, T dL, T pL, T eL, T vxL, T vyL, T vzL, T ByL, T BzL, T dR,
                             T pR, T eR, T vxR, T vyR, T vzR, T ByR, T BzR, T chL, T chR, int jbnd) {
    const FaceSides s = make_sides<T>(Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR,
                                      BzR, chL, chR);
    if (lb.surrogate == SUR_NETWORK) {
      float x[16];
      const float m = face_features(s, x);
#pragma unroll
      for (int k = 0; k < 8; k++) y[k] = m * (lb.norm[32 + k] + y[k] * lb.norm[40 + k]);
    } else if (lb.surrogate == SUR_LLF) {
      llf_outputs(s, y);
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) y[k] = 0.0f;
    }
    flux_from_outputs<T>(s, y, F);
    if (judged) {
      double yt[8];
      face_targets<double>(s, double(gamma), yt);
      double err = 0.0, ref = 0.0, emax = 0.0;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (k == WBX) continue;  // the normal induction flux is exact, not predicted
        const double e = fabs(double(y[k]) - yt[k]);
        err += e;
        ref += fabs(yt[k]);
        emax = fmax(emax, e);
      }
      atomicAdd(&lb.stats[LSTAT_JUDGED], 1.0);
      atomicAdd(&lb.stats[LSTAT_ERR], err);
      atomicAdd(&lb.stats[LSTAT_REF], ref);
      atomicMax(reinterpret_cast<unsigned long long *>(&lb.stats[LSTAT_ERRMAX]),
                (unsigned long long)__double_as_longlong(emax));
    }
    return true;
  }
};

// Positivity of the updated state: the state each cell reaches when this
// face's flux alone is applied over its step (tdt = area times the step)
// keeps at least half of the cell's mass and half of its thermal energy
// (total energy less the kinetic and magnetic parts).  sgn is -1 for the
// cell the flux leaves (s1 side) and +1 for the other.
template <typename R>
__device__ __forceinline__ bool keeps_positive(const LearnBuf &lb, int c, double sgn_tdt, const R *flux) {
  const double *u = lb.U + 10 * (size_t)c;
  const double V = lb.vol[c];
  double a[8], b[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = u[k];
    b[k] = u[k] + sgn_tdt * double(flux[k]);
  }
  auto ethm = [V](const double *q) {
    return q[ENER] - 0.5 * (q[MOMX] * q[MOMX] + q[MOMY] * q[MOMY] + q[MOMZ] * q[MOMZ]) / q[MASS] -
           0.5 * (q[WBX] * q[WBX] + q[WBY] * q[WBY] + q[WBZ] * q[WBZ]) / V;
  };
  if (!(b[MASS] >= 0.5 * a[MASS])) return false;
  return ethm(b) >= 0.5 * ethm(a);
}

}  // namespace fvm
