// Learned face flux inside the rotated-frame flux routine: the compute_flux
// hooks that gate a face, hand it to the network, harvest training pairs,
// and rebuild the flux from the network's output.
//
// The network does not replace the whole flux.  In the frame of the face
// (velocities shifted by the face speed w) the flux is split into the
// central part, the mean of the two sides' physical MHD fluxes, computed
// exactly, and the dissipative remainder of the HLLD solver, which the
// network predicts from 16 features: the side means and jumps of the
// rotated primitives and the two fast speeds, scaled by the mean density
// and the larger fast speed.  The remainder is small on smooth faces, so
// BF16 weights and inputs cost little accuracy there.  The HLLD solution
// is Galilean covariant under a normal boost (mass, momentum, energy and
// induction fluxes transform exactly), so the face-frame flux maps back to
// the moving face's flux without approximation.
//
// Included by fvm_kernels.cu after fvm_math.cuh and flux_mlp.cuh.

namespace fvm {

// Deferred-face buffers, harvest buffers and gate settings of one context.
// The gate: ideal-gas EOS, no boundary neighbour, small relative density and
// pressure jumps, bounded normal Mach number in the face frame, and every
// standardised network input within ZMAX spreads of its training mean.
struct LearnBuf {
  __nv_bfloat16 *X;  // [cap x 16] features of deferred faces
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
  const float *norm; // feature and output standardisation: mu_x[16], 1/sd_x[16], mu_y[8], sd_y[8]
  float drho, dp, mach;  // gate: relative density and pressure jumps, normal Mach number
};
enum { LSTAT_DEFERRED = 0, LSTAT_FALLBACK, LSTAT_JUDGED, LSTAT_ERR, LSTAT_REF, LSTAT_ERRMAX, LSTAT_COUNT = 8 };

__device__ __forceinline__ unsigned face_hash(unsigned f, unsigned salt) {
  unsigned x = f * 0x9E3779B1u ^ (salt * 0x85EBCA77u + 0x165667B1u);
  x ^= x >> 15; x *= 0x2C1B3C6Du; x ^= x >> 12; x *= 0x297A2D39u; x ^= x >> 15;
  return x;
}

// Rotated-frame side states handed to the Riemann hook.
struct FaceSides {
  float Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR, BzR, chL, chR;
};

__device__ __forceinline__ float flux_scale(const FaceSides &s, int k, float rho, float c, float sr) {
  // MASS, MOMX..Z, ENER, WBX..Z
  return k == 0 ? rho * c : (k <= 3 ? rho * c * c : (k == 4 ? rho * c * c * c : sr * c * c));
}

// Physical features of a face (see the file comment).
__device__ __forceinline__ void face_features(const FaceSides &s, float *x) {
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
  const float ic = 1.0f / c, iP = 1.0f / (rho * c * c), iB = 1.0f / (sr * c);
  x[0] = (0.5f * (s.vxL + s.vxR) - s.w) * ic;
  x[1] = 0.5f * (s.vyL + s.vyR) * ic;
  x[2] = 0.5f * (s.vzL + s.vzR) * ic;
  x[3] = 0.5f * (s.pL + s.pR) * iP;
  x[4] = s.Bx * iB;
  x[5] = 0.5f * (s.ByL + s.ByR) * iB;
  x[6] = 0.5f * (s.BzL + s.BzR) * iB;
  x[7] = (s.dR - s.dL) / rho;
  x[8] = (s.vxR - s.vxL) * ic;
  x[9] = (s.vyR - s.vyL) * ic;
  x[10] = (s.vzR - s.vzL) * ic;
  x[11] = (s.pR - s.pL) * iP;
  x[12] = (s.ByR - s.ByL) * iB;
  x[13] = (s.BzR - s.BzL) * iB;
  x[14] = s.chL * ic;
  x[15] = s.chR * ic;
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
__device__ __forceinline__ void central_flux(const FaceSides &s, float *F) {
  float FL[8], FR[8];
  const float sides[2][10] = {{s.dL, s.pL, s.eL, s.vxL - s.w, s.vyL, s.vzL, s.ByL, s.BzL, 0, 0},
                              {s.dR, s.pR, s.eR, s.vxR - s.w, s.vyR, s.vzR, s.ByR, s.BzR, 0, 0}};
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const float d = sides[q][0], p = sides[q][1], e = sides[q][2], u = sides[q][3], v = sides[q][4],
                wz = sides[q][5], by = sides[q][6], bz = sides[q][7], bx = s.Bx;
    const float B2 = bx * bx + by * by + bz * bz;
    const float pT = p + 0.5f * B2;
    const float et = e + 0.5f * (d * (u * u + v * v + wz * wz) + B2);
    float *G = q ? FR : FL;
    G[0] = d * u;
    G[1] = d * u * u + pT - bx * bx;
    G[2] = d * v * u - bx * by;
    G[3] = d * wz * u - bx * bz;
    G[4] = (et + pT) * u - bx * (u * bx + v * by + wz * bz);
    G[5] = 0.0f;
    G[6] = by * u - bx * v;
    G[7] = bz * u - bx * wz;
  }
#pragma unroll
  for (int k = 0; k < 8; k++) F[k] = 0.5f * (FL[k] + FR[k]);
}

// Network targets: the HLLD flux in the face frame minus the central flux,
// scaled (MPI/compute_update.cpp:1109-1341 with w = 0).
__device__ __forceinline__ void face_targets(const FaceSides &s, float gamma, float *y) {
  float Fp[8], Fc[8];
  riemann_hlld<float>(gamma, Fp, s.Bx, 0.0f, s.dL, s.pL, s.eL, s.vxL - s.w, s.vyL, s.vzL, s.ByL, s.BzL, s.dR,
                      s.pR, s.eR, s.vxR - s.w, s.vyR, s.vzR, s.ByR, s.BzR);
  central_flux(s, Fc);
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
#pragma unroll
  for (int k = 0; k < 8; k++) y[k] = (Fp[k] - Fc[k]) / flux_scale(s, k, rho, c, sr);
}

// Rotated lab-frame flux of the moving face from the (unstandardised)
// scaled dissipation y.
template <typename T>
__device__ __forceinline__ void flux_from_outputs(const FaceSides &s, const float *y, T *F) {
  float Fc[8];
  central_flux(s, Fc);
  const float rho = 0.5f * (s.dL + s.dR), c = fmaxf(s.chL, s.chR), sr = sqrtf(rho);
  float Fp[8];
#pragma unroll
  for (int k = 0; k < 8; k++) Fp[k] = Fc[k] + y[k] * flux_scale(s, k, rho, c, sr);
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
  return fabsf(s.dR - s.dL) <= lb.drho * rho && fabsf(s.pR - s.pL) <= lb.dp * pm && fabsf(un) <= lb.mach * c &&
         s.dL > 0.0f && s.dR > 0.0f && s.pL > 0.0f && s.pR > 0.0f;
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
        float x[16], y[8];
        face_features(s, x);
        face_targets(s, float(gamma), y);
#pragma unroll
        for (int k = 0; k < 16; k++) lb.hx[16 * slot + k] = x[k];
#pragma unroll
        for (int k = 0; k < 8; k++) lb.hy[8 * slot + k] = y[k];
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
      o[0] = make_uint4(mlp::pack_bf16(x[0], x[1]), mlp::pack_bf16(x[2], x[3]), mlp::pack_bf16(x[4], x[5]),
                        mlp::pack_bf16(x[6], x[7]));
      o[1] = make_uint4(mlp::pack_bf16(x[8], x[9]), mlp::pack_bf16(x[10], x[11]), mlp::pack_bf16(x[12], x[13]),
                        mlp::pack_bf16(x[14], x[15]));
      lb.gface[slot] = f;
      deferred = true;
      return false;
    }
    riemann_hlld<T>(gamma, F, Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR, BzR);
    return true;
  }
};

// The flux of a deferred face from the network outputs y; one slot in
// lb.judge is also solved exactly and the difference accumulated.
struct LearnedSolver {
  const LearnBuf &lb;
  float *y;  // network output, unstandardised in place
  bool judged;
  template <typename T>
  __device__ bool operator()(T gamma, T *F, T Bx, T w, T dL, T pL, T eL, T vxL, T vyL, T vzL, T ByL, T BzL, T dR,
                             T pR, T eR, T vxR, T vyR, T vzR, T ByR, T BzR, T chL, T chR, int jbnd) {
    const FaceSides s = make_sides<T>(Bx, w, dL, pL, eL, vxL, vyL, vzL, ByL, BzL, dR, pR, eR, vxR, vyR, vzR, ByR,
                                      BzR, chL, chR);
#pragma unroll
    for (int k = 0; k < 8; k++) y[k] = lb.norm[32 + k] + y[k] * lb.norm[40 + k];
    flux_from_outputs<T>(s, y, F);
    if (judged) {
      float yt[8];
      face_targets(s, float(gamma), yt);
      float err = 0.0f, ref = 0.0f, emax = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (k == WBX) continue;  // the normal induction flux is exact, not predicted
        const float e = fabsf(y[k] - yt[k]);
        err += e;
        ref += fabsf(yt[k]);
        emax = fmaxf(emax, e);
      }
      atomicAdd(&lb.stats[LSTAT_JUDGED], 1.0);
      atomicAdd(&lb.stats[LSTAT_ERR], (double)err);
      atomicAdd(&lb.stats[LSTAT_REF], (double)ref);
      atomicMax(reinterpret_cast<unsigned long long *>(&lb.stats[LSTAT_ERRMAX]),
                (unsigned long long)__double_as_longlong((double)emax));
    }
    return true;
  }
};

}  // namespace fvm
