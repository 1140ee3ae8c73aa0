// Host Voronoi mesh builder for periodic boxes (stands in for the CGAL build
// of the reference, MPI/build_mesh_active.cpp:121-851, which this image
// cannot compile).  Each cell is the intersection of the half-spaces
// bounded by the bisector planes of its neighbours; it is computed by
// clipping a convex polyhedron, nearest candidates first, until no farther
// candidate can reach the cell (twice the largest vertex radius).
//
// Output follows the reference's mesh contract (MPI/fvmhd3d.h:169-249):
//   Face { s1, s2, centroid, n }: |n| is the area, n points from s1 to s2,
//         and the centroid is in the periodic frame of s1
//         (|centroid - x_s1| < L/2 per axis);
//   Cell { Volume, centroid, faces }.
// Face area/normal/centroid use the triangle fan about the vertex average
// and the cell volume/centroid the pyramid sum about the generator, the same
// formulas as MPI/build_mesh_active.cpp:474-497 and 563-583; faces with
// sqrt(2*area) < 1e-10 * |centroid - x_i| are dropped
// (MPI/build_mesh_active.cpp:499-501).  Face creation order follows the
// reference: cells are visited in index order and a face is created by the
// first cell that meets it, then appended to both cells' face lists.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

struct V3 {
  double x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  V3 operator+(const V3 &o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3 &o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator*(double s) const { return V3(x * s, y * s, z * s); }
  double dot(const V3 &o) const { return x * o.x + y * o.y + z * o.z; }
  V3 cross(const V3 &o) const { return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
  double norm() const { return std::sqrt(dot(*this)); }
};

struct Poly {            // one face of the clipped cell
  int ngb;               // neighbour cell id, -1 for the bounding box
  V3 u;                  // outward unit normal of the plane
  std::vector<V3> v;     // vertices, counter-clockwise seen from outside
};

struct CellOut {         // per-cell result of the clipping pass
  double vol;
  V3 centroid;           // relative to the generator
  std::vector<int> ngb;
  std::vector<V3> n;     // area-weighted outward normal
  std::vector<V3> c;     // face centroid relative to the generator
  int err;
};

struct Grid {
  int g[3];
  double L[3], h[3];
  std::vector<int> start, idx;
  void build(int n, const double *pos, const double *box) {
    const double spacing = std::cbrt(box[0] * box[1] * box[2] / std::max(n, 1));
    for (int a = 0; a < 3; a++) {
      L[a] = box[a];
      g[a] = std::max(1, (int)std::floor(box[a] / spacing));
      h[a] = box[a] / g[a];
    }
    const size_t ng = (size_t)g[0] * g[1] * g[2];
    std::vector<int> cnt(ng + 1, 0);
    std::vector<int> key(n);
    for (int i = 0; i < n; i++) {
      key[i] = (int)cell_of(pos + 3 * (size_t)i);
      cnt[key[i] + 1]++;
    }
    for (size_t k = 0; k < ng; k++) cnt[k + 1] += cnt[k];
    start = cnt;
    idx.resize(n);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < n; i++) idx[fill[key[i]]++] = i;
  }
  size_t cell_of(const double *p) const {
    int c[3];
    for (int a = 0; a < 3; a++) {
      double x = p[a] - std::floor(p[a] / L[a]) * L[a];
      c[a] = std::min(g[a] - 1, std::max(0, (int)(x / h[a])));
    }
    return ((size_t)c[2] * g[1] + c[1]) * g[0] + c[0];
  }
};

inline double wrap(double d, double L) {
  if (d > 0.5 * L) d -= L;
  else if (d < -0.5 * L) d += L;
  return d;
}

// Clip polyhedron `faces` by the half-space x.u <= off (coordinates relative
// to the generator).  Returns false if nothing was cut.
bool clip(std::vector<Poly> &faces, const V3 &u, double off, int ngb, double tol) {
  bool any_out = false;
  for (size_t f = 0; f < faces.size() && !any_out; f++)
    for (size_t k = 0; k < faces[f].v.size(); k++)
      if (faces[f].v[k].dot(u) - off > tol) { any_out = true; break; }
  if (!any_out) return false;

  std::vector<V3> cap;
  std::vector<Poly> out;
  out.reserve(faces.size() + 1);
  for (size_t f = 0; f < faces.size(); f++) {
    const std::vector<V3> &v = faces[f].v;
    const size_t m = v.size();
    std::vector<V3> nv;
    nv.reserve(m + 2);
    for (size_t k = 0; k < m; k++) {
      const V3 &a = v[k];
      const V3 &b = v[(k + 1) % m];
      const double sa = a.dot(u) - off, sb = b.dot(u) - off;
      const bool ina = sa <= tol, inb = sb <= tol;
      if (ina) nv.push_back(a);
      if (ina != inb) {
        // intersection computed from the inside vertex towards the outside
        // one, so that both faces sharing this edge get the same point
        const V3 &pi = ina ? a : b, &po = ina ? b : a;
        const double si = ina ? sa : sb, so = ina ? sb : sa;
        const double t = si / (si - so);
        const V3 x = pi + (po - pi) * t;
        nv.push_back(x);
        cap.push_back(x);
      }
      if (ina && std::fabs(sa) <= tol) cap.push_back(a);
    }
    // drop consecutive duplicates
    std::vector<V3> cv;
    for (size_t k = 0; k < nv.size(); k++) {
      if (!cv.empty() && (nv[k] - cv.back()).norm() <= tol) continue;
      cv.push_back(nv[k]);
    }
    while (cv.size() > 1 && (cv.front() - cv.back()).norm() <= tol) cv.pop_back();
    if (cv.size() >= 3) {
      Poly p;
      p.ngb = faces[f].ngb;
      p.u = faces[f].u;
      p.v.swap(cv);
      out.push_back(p);
    }
  }
  // cap polygon: unique points on the plane, ordered by angle
  std::vector<V3> pts;
  for (size_t k = 0; k < cap.size(); k++) {
    bool dup = false;
    for (size_t q = 0; q < pts.size(); q++)
      if ((pts[q] - cap[k]).norm() <= tol) { dup = true; break; }
    if (!dup) pts.push_back(cap[k]);
  }
  if (pts.size() >= 3) {
    V3 c;
    for (size_t k = 0; k < pts.size(); k++) c = c + pts[k];
    c = c * (1.0 / pts.size());
    V3 e1 = (std::fabs(u.x) < 0.9) ? V3(1, 0, 0).cross(u) : V3(0, 1, 0).cross(u);
    e1 = e1 * (1.0 / e1.norm());
    const V3 e2 = u.cross(e1);
    std::vector<std::pair<double, int> > ang(pts.size());
    for (size_t k = 0; k < pts.size(); k++) {
      const V3 d = pts[k] - c;
      ang[k] = std::make_pair(std::atan2(d.dot(e2), d.dot(e1)), (int)k);
    }
    std::sort(ang.begin(), ang.end());
    Poly p;
    p.ngb = ngb;
    p.u = u;
    for (size_t k = 0; k < ang.size(); k++) p.v.push_back(pts[ang[k].second]);
    out.push_back(p);
  }
  faces.swap(out);
  return true;
}

void build_cell(int i, int n, const double *pos, const Grid &G, double tol_rel, CellOut &res) {
  res.err = 0;
  const double *pi = pos + 3 * (size_t)i;
  const double hmax = std::max(G.h[0], std::max(G.h[1], G.h[2]));
  const double tol = tol_rel * hmax;
  // initial box: half the periodic box in every direction
  const double B[3] = {0.5 * G.L[0], 0.5 * G.L[1], 0.5 * G.L[2]};
  std::vector<Poly> faces(6);
  const V3 corner[8] = {V3(-B[0], -B[1], -B[2]), V3(B[0], -B[1], -B[2]), V3(B[0], B[1], -B[2]),
                        V3(-B[0], B[1], -B[2]), V3(-B[0], -B[1], B[2]), V3(B[0], -B[1], B[2]),
                        V3(B[0], B[1], B[2]), V3(-B[0], B[1], B[2])};
  const int quad[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 4, 7, 3}, {1, 2, 6, 5}};
  const V3 un[6] = {V3(0, 0, -1), V3(0, 0, 1), V3(0, -1, 0), V3(0, 1, 0), V3(-1, 0, 0), V3(1, 0, 0)};
  for (int f = 0; f < 6; f++) {
    faces[f].ngb = -1;
    faces[f].u = un[f];
    for (int k = 0; k < 4; k++) faces[f].v.push_back(corner[quad[f][k]]);
  }

  int c0[3];
  {
    size_t key = G.cell_of(pi);
    c0[0] = (int)(key % G.g[0]);
    c0[1] = (int)((key / G.g[0]) % G.g[1]);
    c0[2] = (int)(key / ((size_t)G.g[0] * G.g[1]));
  }
  const int kmax = std::max(G.g[0], std::max(G.g[1], G.g[2])) / 2;
  std::vector<std::pair<double, std::pair<int, V3> > > cand;
  for (int shell = 0; shell <= kmax; shell++) {
    cand.clear();
    for (int dz = -shell; dz <= shell; dz++)
      for (int dy = -shell; dy <= shell; dy++)
        for (int dx = -shell; dx <= shell; dx++) {
          if (std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz))) != shell) continue;
          if (2 * shell + 1 > G.g[0] && std::abs(dx) > G.g[0] / 2) continue;
          if (2 * shell + 1 > G.g[1] && std::abs(dy) > G.g[1] / 2) continue;
          if (2 * shell + 1 > G.g[2] && std::abs(dz) > G.g[2] / 2) continue;
          const int cx = ((c0[0] + dx) % G.g[0] + G.g[0]) % G.g[0];
          const int cy = ((c0[1] + dy) % G.g[1] + G.g[1]) % G.g[1];
          const int cz = ((c0[2] + dz) % G.g[2] + G.g[2]) % G.g[2];
          const size_t key = ((size_t)cz * G.g[1] + cy) * G.g[0] + cx;
          for (int q = G.start[key]; q < G.start[key + 1]; q++) {
            const int j = G.idx[q];
            if (j == i) continue;
            const double *pj = pos + 3 * (size_t)j;
            const V3 d(wrap(pj[0] - pi[0], G.L[0]), wrap(pj[1] - pi[1], G.L[1]), wrap(pj[2] - pi[2], G.L[2]));
            cand.push_back(std::make_pair(d.dot(d), std::make_pair(j, d)));
          }
        }
    std::sort(cand.begin(), cand.end(),
              [](const std::pair<double, std::pair<int, V3> > &a, const std::pair<double, std::pair<int, V3> > &b) {
                return a.first < b.first || (a.first == b.first && a.second.first < b.second.first);
              });
    for (size_t k = 0; k < cand.size(); k++) {
      const V3 &d = cand[k].second.second;
      const double dn = std::sqrt(cand[k].first);
      clip(faces, d * (1.0 / dn), 0.5 * dn, cand[k].second.first, tol);
    }
    // security radius: every point not yet seen is at least shell*h away
    double r2max = 0.0;
    for (size_t f = 0; f < faces.size(); f++)
      for (size_t k = 0; k < faces[f].v.size(); k++) r2max = std::max(r2max, faces[f].v[k].dot(faces[f].v[k]));
    const double hmin = std::min(G.h[0], std::min(G.h[1], G.h[2]));
    if (2.0 * std::sqrt(r2max) < shell * hmin) break;
    if (shell == kmax) { res.err = 1; }
  }

  // face geometry and cell volume (reference formulas, relative coordinates)
  res.vol = 0.0;
  res.centroid = V3();
  V3 csum;
  double vsum = 0.0;
  for (size_t f = 0; f < faces.size(); f++) {
    const Poly &p = faces[f];
    if (p.ngb < 0) { res.err = 2; continue; }
    const size_t m = p.v.size();
    V3 c;
    for (size_t k = 0; k < m; k++) c = c + p.v[k];
    c = c * (1.0 / (double)m);
    V3 fn, fc;
    double area1 = 0.0;
    V3 v1 = p.v[m - 1] - c;
    const double third = 1.0 / 3.0;
    for (size_t k = 0; k < m; k++) {
      const V3 v2 = p.v[k] - c;
      const V3 n3 = v1.cross(v2);
      const double a3 = n3.norm();
      fn = fn + n3;
      fc = fc + (c + (v1 + v2) * third) * a3;
      area1 += a3;
      v1 = v2;
    }
    if (!(area1 > 0.0)) continue;
    fc = fc * (1.0 / area1);
    if (std::sqrt(area1) < 1.0e-10 * fc.norm()) continue;
    fn = fn * 0.5;
    if (fn.norm() == 0.0) continue;
    if (fc.dot(fn) < 0.0) fn = fn * -1.0;
    // a cell may meet each neighbour once: two faces with the same neighbour
    // mean the cell spans more than half the periodic box
    for (size_t q = 0; q < res.ngb.size(); q++)
      if (res.ngb[q] == p.ngb) res.err |= 4;
    res.ngb.push_back(p.ngb);
    res.n.push_back(fn);
    res.c.push_back(fc);
    // pyramid about the generator, apex at the origin
    const V3 cv = fc * -1.0;
    V3 w1 = p.v[m - 1] - fc;
    for (size_t k = 0; k < m; k++) {
      const V3 w2 = p.v[k] - fc;
      const V3 c4 = fc + (w1 + w2 + cv) * 0.25;
      const double v4 = std::fabs(w1.cross(w2).dot(cv));
      vsum += v4;
      csum = csum + c4 * v4;
      w1 = w2;
    }
  }
  res.centroid = vsum > 0.0 ? csum * (1.0 / vsum) : V3();
  res.vol = vsum / 6.0;
  (void)n;
}

struct Mesh {
  int ncell;
  std::vector<int> s1, s2;
  std::vector<double> fn, fc;           // 3 per face
  std::vector<double> vol, cc;          // per cell
  std::vector<std::vector<int> > cf;    // face ids per cell
  int err;
};

}  // namespace

extern "C" {

// Builds the periodic Voronoi mesh of n generators in [0,box)^3.
// Returns an opaque handle (NULL on allocation failure).  nthreads <= 0
// uses the OpenMP default.
void *fvm_mesh_build(int n, const double *pos, const double *box, int nthreads) {
  Mesh *M = new Mesh;
  M->ncell = n;
  M->err = 0;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Grid G;
  G.build(n, pos, box);
  M->vol.assign(n, 0.0);
  M->cc.assign(3 * (size_t)n, 0.0);
  M->cf.assign(n, std::vector<int>());
  const int chunk = 1 << 16;
  std::vector<CellOut> res;
  for (int base = 0; base < n; base += chunk) {
    const int m = std::min(chunk, n - base);
    res.assign(m, CellOut());
    int err = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : err)
    for (int k = 0; k < m; k++) {
      build_cell(base + k, n, pos, G, 1.0e-13, res[k]);
      err |= res[k].err;
    }
    M->err |= err;
    for (int k = 0; k < m; k++) {
      const int i = base + k;
      const CellOut &r = res[k];
      M->vol[i] = r.vol;
      for (int a = 0; a < 3; a++) M->cc[3 * (size_t)i + a] = pos[3 * (size_t)i + a] + (&r.centroid.x)[a];
      for (size_t f = 0; f < r.ngb.size(); f++) {
        const int j = r.ngb[f];
        bool found = false;
        for (size_t q = 0; q < M->cf[i].size(); q++) {
          const int fid = M->cf[i][q];
          const int other = M->s1[fid] == i ? M->s2[fid] : M->s1[fid];
          if (other == j) { found = true; break; }
        }
        if (found) continue;
        const int fid = (int)M->s1.size();
        M->s1.push_back(i);
        M->s2.push_back(j);
        for (int a = 0; a < 3; a++) {
          M->fn.push_back((&r.n[f].x)[a]);
          M->fc.push_back(pos[3 * (size_t)i + a] + (&r.c[f].x)[a]);
        }
        M->cf[i].push_back(fid);
        M->cf[j].push_back(fid);
      }
    }
  }
  return M;
}

int fvm_mesh_error(void *h) { return ((Mesh *)h)->err; }

void fvm_mesh_sizes(void *h, int *nface, long long *nlink) {
  Mesh *M = (Mesh *)h;
  *nface = (int)M->s1.size();
  long long s = 0;
  for (int i = 0; i < M->ncell; i++) s += (long long)M->cf[i].size();
  *nlink = s;
}

void fvm_mesh_fetch(void *h, int *s1, int *s2, double *fn, double *fc, double *vol, double *cc,
                    long long *off, int *ids) {
  Mesh *M = (Mesh *)h;
  const size_t nf = M->s1.size();
  memcpy(s1, M->s1.data(), nf * sizeof(int));
  memcpy(s2, M->s2.data(), nf * sizeof(int));
  memcpy(fn, M->fn.data(), 3 * nf * sizeof(double));
  memcpy(fc, M->fc.data(), 3 * nf * sizeof(double));
  memcpy(vol, M->vol.data(), (size_t)M->ncell * sizeof(double));
  memcpy(cc, M->cc.data(), 3 * (size_t)M->ncell * sizeof(double));
  long long o = 0;
  for (int i = 0; i < M->ncell; i++) {
    off[i] = o;
    for (size_t q = 0; q < M->cf[i].size(); q++) ids[o++] = M->cf[i][q];
  }
  off[M->ncell] = o;
}

void fvm_mesh_free(void *h) { delete (Mesh *)h; }

}  // extern "C"
