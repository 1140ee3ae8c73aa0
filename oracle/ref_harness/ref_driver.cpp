/*
 * Harness that drives the reference's own MPI-tree hot path, compiled
 * unmodified from its sources, on one rank.  TEST INFRASTRUCTURE ONLY: the
 * resulting library (oracle/_ref/libfvmref.so) is the checker that pins the
 * plain-C oracle and the GPU path; nothing in the product links it.
 *
 * What the harness supplies (everything else is the reference's code):
 *   - the problem hooks the reference leaves to its problem files
 *     (ideal gas: MPI/set_problem.cpp:89-137; isothermal disk:
 *     MPI/problems/mri_disk3d.cpp:359-389);
 *   - a mesh installer that stands in for the CGAL build
 *     (MPI/build_mesh_active.cpp:663-851): it copies a precomputed Voronoi
 *     mesh into cell_list/face_list and sets the site flags the way
 *     MPI/build_mesh_active.cpp:524-528 does;
 *   - a one-rank step driver that follows system::iterate_step
 *     (MPI/iterate.cpp:115-247) minus the meshing and domain decomposition,
 *     with an optional "shared" mode that puts every cell on the rung of the
 *     global minimum timestep (the effect of compute_timesteps(true),
 *     MPI/compute_timestep.cpp:57-75).
 *
 * compute_update.cpp is compiled by inclusion in this translation unit so that
 * its inline system::compute_flux can be called directly for per-face
 * known-answer checks.
 */
#include "compute_update.cpp"

#include <vector>
#include <algorithm>

namespace fvm_mpi_stub {
  int type_size[NTYPE];
  int ntype = 0;
}


/* ---- problem hooks ------------------------------------------------------ */

namespace {
  int    g_eos = 0;          /* 0: ideal gas, 1: isothermal disk */
  double g_iso_GM = 1.0;     /* disk: cs^2(r) = GM/|r| * c_fac^2 */
  double g_iso_cfac = 0.05;
  int    g_static_mesh = 0;  /* 1: static generators */
}

namespace fvmhd3d {

  bool system::problem_force_distribute() { return false; }
  /* The reference's default hook returns false (MPI/set_problem.cpp:61-76);
   * its disabled branch, used here for static generators, zeroes vel of every
   * active site and returns true. */
  bool system::compute_pvel1()
  {
    if (!g_static_mesh) return false;
    for (size_t a = 0; a < site_active_list.size(); a++) ptcl_import[site_active_list[a]].vel = 0.0;
    return true;
  }

  /* MPI/set_problem.cpp:77-87 */
  void system::predict(const int i)
  {
    Particle &p = ptcl_local[i];
    p.acc0 = p.acc1 = 0.0;
    const real dt = t_global - p.tlast;
    p.vel = p.orig_vel;
    p.pos = p.orig_pos + p.orig_vel*dt;
  }

  /* MPI/set_problem.cpp:89-101 */
  void system::correct(const int i0)
  {
    const int i = i0 < 0 ? -1-i0 : i0;
    Particle &p = ptcl_local[i];
    const real dth = 0.5*(t_global - p.tlast);
    p.orig_pos = p.orig_pos + (p.vel + p.orig_vel)*dth;
    p.orig_vel = p.vel;
    p.pot = 0.0;
    p.tlast = scheduler.get_tsys();
    p.tend  = scheduler.get_tsys() + scheduler.get_dt(p.rung);
  }

  /* ideal gas: MPI/set_problem.cpp:102-105; disk: mri_disk3d.cpp:359-365 */
  const real system::extra_timestep(const int i)
  {
    if (g_eos == 0) return HUGE;
    const Particle &p = ptcl_import[i];
    if (p.is_boundary()) return HUGE;
    const real r = p.pos.abs();
    return courant_no*r/(1.0/HUGE + p.vel.abs());
  }

  bool system::compute_update_prob(Fluid &, const int) { return false; }

  real system::compute_ethm_update(const Fluid &W, const int i) const
  {
    if (g_eos == 0) return W[Fluid::ETHM];
    const real r = ptcl_import[i].pos.abs();
    return (g_iso_GM/r)*sqr(g_iso_cfac)*W[Fluid::DENS];
  }
  real system::compute_pressure(const Fluid &W) const
  {
    if (g_eos == 0) return gamma_gas > 1.0 ? (gamma_gas - 1.0) * W[Fluid::ETHM] : W[Fluid::ETHM];
    return W[Fluid::ETHM];
  }
  real system::compute_entropy_from_ethm(const Fluid &W) const
  {
    if (g_eos == 0) return (gamma_gas - 1.0) * W[Fluid::ETHM]/std::pow(W[Fluid::DENS], gamma_gas);
    return 1.0;
  }
  real system::compute_ethm_from_entropy(const Fluid &W) const
  {
    if (g_eos == 0) return W[Fluid::ENTR] * std::pow(W[Fluid::DENS], gamma_gas)/(gamma_gas - 1.0);
    abort();
    return -1.0;
  }

  void system::distribute_data(const bool, const bool, const bool)
  {
    fprintf(stderr, "ref harness: distribute_data is not reachable on one rank\n");
    abort();
  }

  /* The CGAL mesh build is replaced by install_mesh() below; iterate_step,
   * its only caller, is not used by this harness. */
  void system::build_mesh_active(std::vector<int> &, std::vector< std::vector<int> > &,
                                 std::vector<int> &)
  {
    fprintf(stderr, "ref harness: build_mesh_active needs CGAL; use install_mesh\n");
    abort();
  }
}

/* ---- C-ABI --------------------------------------------------------------- */

using namespace fvmhd3d;
typedef fvmhd3d::system fsys;

struct ref_params {
  double gamma, courant;
  double box[3];
  double dtmax;
  int    eos;
  double iso_GM, iso_cfac;
  int    static_mesh;
};

struct ref_snap {
  double *wrec_after_limiter;    /* ncell*50 */
  double *U_after_update;        /* ncell*10 */
  double *dU_after_update;       /* ncell*14 */
  double *vel_after_pvel;        /* ncell*3  */
  int    *rung_after_timestep;   /* ncell    */
  double *dt_after_timestep;     /* ncell (left untouched: see ref_step) */
  double *wrec_after_update0;    /* ncell*50 */
  int    *rung_after_update0;    /* ncell    */
  double *wrec_after_recon;      /* ncell*50 */
  int    *active_faces;          /* nface (face ids, order of face_active_list) */
  int    *nactive_faces;         /* 1 */
};

struct RefCtx {
  fsys *s;
  int ncell, nface;
  std::vector<Face> faces;
  std::vector<Cell> cells;
};

static void install_mesh(RefCtx *c)
{
  fsys &s = *c->s;
  const int n = c->ncell;
  s.cell_list = c->cells;
  s.face_list = c->faces;
  s.site_import.clear();
  s.site_active_list.clear();
  s.site_with_ngb_active_list.clear();
  for (int i = 0; i < n; i++)
  {
    s.site_import.push_back(SiteImport(s.ptcl_local[i].pos, 0, i, 0.0));
    if (s.ptcl_local[i].is_active()) s.site_import[i].set_active();
  }
  for (int i = 0; i < n; i++)
  {
    if (!s.site_import[i].is_active()) continue;
    s.site_active_list.push_back(i);
    const Cell &ci = s.cell_list[i];
    for (int k = 0; k < (int)ci.ngb.size(); k++)
    {
      const int j = s.face_list[ci.ngb[k]].ngb<false>(i);
      if (!s.site_import[j].is_active())
      {
        s.site_import[j].set_local_ngb();
        s.site_import[i].set_hasngb();
      }
    }
  }
}

static void clear_import(fsys &s)
{
  clear_vec(s.cell_list);
  clear_vec(s.face_list);
  clear_vec(s.ptcl_import);
  clear_vec(s.U_import);
  clear_vec(s.dU_import);
  clear_vec(s.Wrec_import);
  clear_vec(s.Wst_import);
  clear_vec(s.Wextra_import);
}

static void copy_wrec(const fsys &s, double *out)
{
  if (!out) return;
  const int n = s.Wrec_import.size();
  for (int i = 0; i < n; i++)
  {
    const Fluid_rec &r = s.Wrec_import[i];
    for (int k = 0; k < 10; k++)
    {
      out[i*50 +  0 + k] = r.w[k];
      out[i*50 + 10 + k] = r.x[k];
      out[i*50 + 20 + k] = r.y[k];
      out[i*50 + 30 + k] = r.z[k];
      out[i*50 + 40 + k] = r.t[k];
    }
  }
}

extern "C" {

void *ref_create(const ref_params *p)
{
  RefCtx *c = new RefCtx;
  c->s = new fsys(0, 1);
  c->ncell = c->nface = 0;
  fsys &s = *c->s;
  s.gamma_gas  = p->gamma;
  s.courant_no = p->courant;
  s.global_domain_size = vec3(p->box[0], p->box[1], p->box[2]);
  s.global_domain = boundary(vec3(0.0), s.global_domain_size);
  s.scheduler = Scheduler(p->dtmax);
  s.t_global = 0.0;
  g_eos = p->eos;
  g_iso_GM = p->iso_GM;
  g_iso_cfac = p->iso_cfac;
  g_static_mesh = p->static_mesh;
  return c;
}

void ref_destroy(void *h)
{
  RefCtx *c = (RefCtx *)h;
  delete c->s;
  delete c;
}

int ref_set_mesh(void *h, int ncell, int nface,
                 const int *s1, const int *s2, const double *fn, const double *fc,
                 const double *cvol, const double *cc, const int *off, const int *ids)
{
  RefCtx *c = (RefCtx *)h;
  c->ncell = ncell;
  c->nface = nface;
  c->faces.resize(nface);
  for (int f = 0; f < nface; f++)
  {
    c->faces[f].s1 = s1[f];
    c->faces[f].s2 = s2[f];
    c->faces[f].n = vec3(fn[3*f], fn[3*f+1], fn[3*f+2]);
    c->faces[f].centroid = vec3(fc[3*f], fc[3*f+1], fc[3*f+2]);
  }
  c->cells.clear();
  c->cells.resize(ncell);
  for (int i = 0; i < ncell; i++)
  {
    c->cells[i].Volume = cvol[i];
    c->cells[i].centroid = vec3(cc[3*i], cc[3*i+1], cc[3*i+2]);
    for (int k = off[i]; k < off[i+1]; k++) c->cells[i].ngb.push_back(ids[k]);
  }
  return 0;
}

/* Initial state, following the tail of the reference's set_problem
 * (MPI/problems/mri_disk3d.cpp:832-880): W -> Wrec=(W,0,0,0,0), U = W->cons,
 * dU = 0, then compute_pvel + compute_timesteps(true) on all cells, rung +=
 * rung_offset, tend = dt(rung), and every cell pushed to its rung list. */
int ref_init_problem(void *h, const double *W, const double *pos, const int *bnd, int rung_offset)
{
  RefCtx *c = (RefCtx *)h;
  fsys &s = *c->s;
  const int n = c->ncell;
  s.local_n = s.global_n = n;
  s.ptcl_local.assign(n, Particle());
  s.U_local.resize(n);
  s.dU_local.assign(n, FluidD(0.0));
  s.Wrec_local.resize(n);
  s.divBi.assign(n, 0.0f);
  s.Wextra_local.resize(n);
  for (int i = 0; i < n; i++) s.Wextra_local[i].J = vec3(0.0);
  s.ngb_list.assign(n, Neighbours<Ngb>());
  for (int i = 0; i < n; i++)
  {
    Particle &p = s.ptcl_local[i];
    p.set_pos(vec3(pos[3*i], pos[3*i+1], pos[3*i+2]));
    p.vel = p.orig_vel = vec3(0.0);
    p.acc0 = p.acc1 = vec3(0.0);
    p.tlast = 0.0;
    p.tend = 0.0;
    p.rung = 0;
    p.boundary = bnd ? bnd[i] : 0;
    p.idx = i;
    p.rmax = 0.0f;
    p.local_id = i;
    p.volume = p.volume_new = c->cells[i].Volume;
    Fluid m;
    for (int k = 0; k < 10; k++) m[k] = W[10*i + k];
    s.Wrec_local[i] = Fluid_rec(m);
    s.U_local[i] = m.to_conservative(c->cells[i].Volume);
  }
  s.get_active_ptcl(true);
  s.cell_list = c->cells;
  s.face_list = c->faces;
  s.U_import.swap(s.U_local);
  s.ptcl_import.swap(s.ptcl_local);
  s.site_active_list.swap(s.active_ptcl);
  s.compute_pvel();
  s.compute_timesteps(true);
  s.U_import.swap(s.U_local);
  s.ptcl_import.swap(s.ptcl_local);
  s.site_active_list.swap(s.active_ptcl);
  clear_vec(s.cell_list);
  clear_vec(s.face_list);
  for (int i = 0; i < n; i++)
  {
    s.ptcl_local[i].rung += rung_offset;
    s.ptcl_local[i].tend = 0.0 + s.scheduler.get_dt(s.ptcl_local[i].rung);
    s.ptcl_local[i].orig_vel = s.ptcl_local[i].vel;
  }
  s.scheduler.flush_list();
  for (int i = 0; i < n; i++)
  {
    s.scheduler.push_particle(i, (int)s.ptcl_local[i].rung);
    s.ptcl_local[i].unset_active();
  }
  return 0;
}

/* One iterate_step (MPI/iterate.cpp:115-247) on the installed mesh. */
int ref_step(void *h, int shared, ref_snap *snap)
{
  RefCtx *c = (RefCtx *)h;
  fsys &s = *c->s;
  s.iteration++;
  s.get_active_ptcl(false);
  install_mesh(c);
  s.distribute_particle_fluid_data();
  s.get_active_faces();
  if (snap && snap->nactive_faces) *snap->nactive_faces = s.nface_active;
  if (snap && snap->active_faces)
    for (int f = 0; f < s.nface_active; f++)
      snap->active_faces[f] = (int)(s.face_active_list[f] - &s.face_list[0]);

  /* fluid_update(true), MPI/iterate.cpp:97-107, with snapshots between stages */
  s.slope_limiter();
  if (snap) copy_wrec(s, snap->wrec_after_limiter);
  s.compute_update();
  if (snap && snap->U_after_update)
    for (int i = 0; i < c->ncell; i++)
      for (int k = 0; k < 10; k++) snap->U_after_update[10*i+k] = s.U_import[i][k];
  if (snap && snap->dU_after_update)
    for (int i = 0; i < c->ncell; i++)
    {
      for (int k = 0; k < 10; k++) snap->dU_after_update[14*i+k] = s.dU_import[i].U[k];
      snap->dU_after_update[14*i+10] = s.dU_import[i].gradPsi.x;
      snap->dU_after_update[14*i+11] = s.dU_import[i].gradPsi.y;
      snap->dU_after_update[14*i+12] = s.dU_import[i].gradPsi.z;
      snap->dU_after_update[14*i+13] = s.dU_import[i].divB;
    }
  s.compute_pvel();
  if (snap && snap->vel_after_pvel)
    for (int i = 0; i < c->ncell; i++)
    {
      snap->vel_after_pvel[3*i+0] = s.ptcl_import[i].vel.x;
      snap->vel_after_pvel[3*i+1] = s.ptcl_import[i].vel.y;
      snap->vel_after_pvel[3*i+2] = s.ptcl_import[i].vel.z;
    }
  s.compute_timesteps(false);
  if (snap && snap->rung_after_timestep)
    for (int i = 0; i < c->ncell; i++) snap->rung_after_timestep[i] = s.ptcl_import[i].rung;
  /* dt_after_timestep is not available here: the reference keeps the
   * per-cell dt in a vector local to compute_timesteps
   * (MPI/compute_timestep.cpp:81,97). */

  if (shared)
  {
    int rmax = 0;
    for (size_t a = 0; a < s.site_active_list.size(); a++)
      rmax = std::max(rmax, s.ptcl_import[s.site_active_list[a]].rung);
    for (size_t a = 0; a < s.site_active_list.size(); a++)
      s.ptcl_import[s.site_active_list[a]].rung = rmax;
  }

  s.collect_results();
  s.distribute_fluid_update_data();

  /* fluid_update(false), MPI/iterate.cpp:108-112 */
  s.compute_update0();
  if (snap) copy_wrec(s, snap->wrec_after_update0);
  if (snap && snap->rung_after_update0)
    for (int i = 0; i < c->ncell; i++) snap->rung_after_update0[i] = s.ptcl_import[i].rung;
  s.compute_reconstruction();
  if (snap) copy_wrec(s, snap->wrec_after_recon);

  s.collect_reconstruction();

  if (shared)
  {
    int rmax = 0;
    for (size_t a = 0; a < s.active_ptcl.size(); a++)
      rmax = std::max(rmax, s.ptcl_local[s.active_ptcl[a]].rung);
    for (size_t a = 0; a < s.active_ptcl.size(); a++)
    {
      Particle &p = s.ptcl_local[s.active_ptcl[a]];
      p.rung = rmax;
      p.tend = s.t_global + s.scheduler.get_dt(rmax);
    }
  }

  /* rung re-insertion, MPI/iterate.cpp:199-217 */
  for (size_t a = 0; a < s.active_ptcl.size(); a++)
  {
    const int i = s.active_ptcl[a];
    s.scheduler.push_particle(i, (int)s.ptcl_local[i].rung);
    s.ptcl_local[i].unset_active();
  }
  clear_import(s);
  return (int)s.active_ptcl.size();
}

double ref_time(void *h) { return ((RefCtx *)h)->s->t_global; }

/* orig_pos / orig_vel of the particles and divBi (after a step). */
int ref_get_motion(void *h, double *opos, double *ovel, float *divb)
{
  RefCtx *c = (RefCtx *)h;
  fsys &s = *c->s;
  for (int i = 0; i < c->ncell; i++)
  {
    const Particle &p = s.ptcl_local[i];
    if (opos) { opos[3*i] = p.orig_pos.x; opos[3*i+1] = p.orig_pos.y; opos[3*i+2] = p.orig_pos.z; }
    if (ovel) { ovel[3*i] = p.orig_vel.x; ovel[3*i+1] = p.orig_vel.y; ovel[3*i+2] = p.orig_vel.z; }
    if (divb) divb[i] = s.divBi[i];
  }
  return 0;
}

/* The reference's snapshot writer, system::dump_binary (MPI/dump_binary.cpp). */
int ref_dump_binary(void *h, const char *path)
{
  RefCtx *c = (RefCtx *)h;
  c->s->dump_binary(path);
  return 0;
}
double ref_dt_tick(void *h) { return ((RefCtx *)h)->s->scheduler.dt_tick; }
unsigned long long ref_tsys_ticks(void *h) { return ((RefCtx *)h)->s->scheduler.tsysU; }

/* Full per-cell state of the local arrays (between steps). */
int ref_get_state(void *h, double *pos, double *vel, double *tlast, double *tend,
                  int *rung, double *U, double *dU, double *wrec)
{
  RefCtx *c = (RefCtx *)h;
  fsys &s = *c->s;
  for (int i = 0; i < c->ncell; i++)
  {
    const Particle &p = s.ptcl_local[i];
    if (pos)   { pos[3*i] = p.pos.x; pos[3*i+1] = p.pos.y; pos[3*i+2] = p.pos.z; }
    if (vel)   { vel[3*i] = p.vel.x; vel[3*i+1] = p.vel.y; vel[3*i+2] = p.vel.z; }
    if (tlast) tlast[i] = p.tlast;
    if (tend)  tend[i] = p.tend;
    if (rung)  rung[i] = p.rung;
    if (U) for (int k = 0; k < 10; k++) U[10*i+k] = s.U_local[i][k];
    if (dU)
    {
      for (int k = 0; k < 10; k++) dU[14*i+k] = s.dU_local[i].U[k];
      dU[14*i+10] = s.dU_local[i].gradPsi.x;
      dU[14*i+11] = s.dU_local[i].gradPsi.y;
      dU[14*i+12] = s.dU_local[i].gradPsi.z;
      dU[14*i+13] = s.dU_local[i].divB;
    }
    if (wrec)
      for (int k = 0; k < 10; k++)
      {
        const Fluid_rec &r = s.Wrec_local[i];
        wrec[i*50 +  0 + k] = r.w[k];
        wrec[i*50 + 10 + k] = r.x[k];
        wrec[i*50 + 20 + k] = r.y[k];
        wrec[i*50 + 30 + k] = r.z[k];
        wrec[i*50 + 40 + k] = r.t[k];
      }
  }
  return 0;
}

/* Per-face known-answer entry: system::compute_flux on given face states. */
int ref_compute_flux(void *h, int nface, const double *wij, const double *Wi, const double *Wj,
                     const int *jbnd, const double *normal, double *psi, double *Bn, double *flux)
{
  RefCtx *c = (RefCtx *)h;
  fsys &s = *c->s;
  for (int f = 0; f < nface; f++)
  {
    Fluid a, b, F;
    for (int k = 0; k < 10; k++) { a[k] = Wi[10*f+k]; b[k] = Wj[10*f+k]; }
    real p, bn;
    s.compute_flux(vec3(wij[3*f], wij[3*f+1], wij[3*f+2]), a, b, jbnd ? jbnd[f] : 0,
                   vec3(normal[3*f], normal[3*f+1], normal[3*f+2]), p, bn, F);
    psi[f] = p;
    Bn[f] = bn;
    for (int k = 0; k < 10; k++) flux[10*f+k] = F[k];
  }
  return 0;
}

} /* extern "C" */
