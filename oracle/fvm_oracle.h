/*
 * Plain-C restatement of fvmhd3d's per-timestep fluid hot path (MPI tree),
 * one rank, periodic mesh given as arrays.  TEST INFRASTRUCTURE ONLY: this
 * is the oracle the CUDA path is checked against; the product never links
 * it.  Each function cites the reference lines it restates.
 *
 * Layouts (all row-major, one record per cell or face):
 *   face:  s1, s2 (int32); n[3] (area-weighted normal s1->s2); c[3] (face
 *          centroid in the frame of s1)
 *   cell:  volume; face ids in CSR form (off[ncell+1] int64, ids int32)
 *   state: pos[3], vel[3] (mesh-generator velocity), tlast, tend, rung,
 *          bnd, U[10] (conserved), dU[14] (accumulated dU[10], gradPsi[3],
 *          divB), Wrec[50] (w, x, y, z, t blocks of 10 primitives)
 */
#ifndef FVM_ORACLE_H
#define FVM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fvo_params {
  double gamma, courant;
  double box[3];
  double dtmax;
  int eos;                 /* 0 ideal gas, 1 isothermal disk */
  double iso_GM, iso_cfac; /* disk: cs^2 = GM/|r| * cfac^2 */
  int static_mesh;         /* 1: compute_pvel1 hook with vel = 0 (MPI/set_problem.cpp:61-72) */
} fvo_params;

/* snapshots between stages of one step (any pointer may be NULL) */
typedef struct fvo_snap {
  double *wrec_after_limiter;  /* ncell*50 */
  double *U_after_update;      /* ncell*10 */
  double *dU_after_update;     /* ncell*14 */
  double *vel_after_pvel;      /* ncell*3 */
  int *rung_after_timestep;    /* ncell */
  double *dt_after_timestep;   /* ncell */
  double *wrec_after_update0;  /* ncell*50 */
  int *rung_after_update0;     /* ncell */
  double *wrec_after_recon;    /* ncell*50 */
  int *active_faces;           /* nface */
  int *nactive_faces;          /* 1 */
} fvo_snap;

typedef struct fvo_ctx fvo_ctx;

fvo_ctx *fvo_create(const fvo_params *p);
void fvo_destroy(fvo_ctx *c);
int fvo_set_mesh(fvo_ctx *c, int ncell, int nface, const int *s1, const int *s2,
                 const double *fn, const double *fc, const double *cvol, const double *cc,
                 const long long *off, const int *ids);
int fvo_init_problem(fvo_ctx *c, const double *W, const double *pos, const int *bnd, int rung_offset);
int fvo_step(fvo_ctx *c, int shared, fvo_snap *snap);
double fvo_time(const fvo_ctx *c);
int fvo_clock(const fvo_ctx *c, unsigned long long *tsys, double *dt_global, long long *iteration);
int fvo_get_motion(const fvo_ctx *c, double *opos, double *ovel, float *divb);
int fvo_get_state(const fvo_ctx *c, double *pos, double *vel, double *tlast, double *tend,
                  int *rung, double *U, double *dU, double *wrec);
int fvo_set_state(fvo_ctx *c, const double *vel, const double *tlast, const double *tend,
                  const int *rung, const double *U, const double *dU, const double *wrec,
                  unsigned long long tsys_ticks);
int fvo_compute_flux(const fvo_ctx *c, int nface, const double *wij, const double *Wi,
                     const double *Wj, const int *jbnd, const double *normal,
                     double *psi, double *Bn, double *flux);

#ifdef __cplusplus
}
#endif
#endif
