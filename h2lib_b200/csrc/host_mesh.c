/* Host-side surface meshes: macro surfaces (sphere, cube), uniform refinement and the
 * per-triangle normals / Gram determinants the quadrature consumes.
 *
 * Restates, in this project's own code:
 *   new_sphere_macrosurface3d        Library/macrosurface3d.c:81   (octahedron projected to S^2)
 *   new_cube_macrosurface3d          Library/macrosurface3d.c:390  (= cuboid [-1,1]^3, :264)
 *   build_from_macrosurface3d_surface3d Library/macrosurface3d.c:707 (split^2 refinement)
 *   prepare_surface3d                Library/surface3d.c:51        (n, g = 2*area, hmin/hmax)
 * The macro vertex/edge/triangle tables and the order in which refined vertices and triangles are
 * numbered must match the reference exactly (index-for-index), otherwise matrices assembled on the
 * same "sphere split 64" would not be comparable entry by entry.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "h2b200_internal.h"

typedef struct {
  uint32_t nv, ne, nt;
  const double (*x)[3];
  const uint32_t (*e)[2];
  const uint32_t (*t)[3];
  const uint32_t (*s)[3];   /* macro edge opposite to local vertex j of triangle i */
  int project_to_sphere;
} macro_t;

/* Octahedron: vertices front(+z), right(+x), back(-z), left(-x), top(+y), bottom(-y). */
static const double sphere_x[6][3] = {
  {0, 0, 1}, {1, 0, 0}, {0, 0, -1}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
static const uint32_t sphere_e[12][2] = {
  {0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 4}, {2, 4}, {3, 4}, {0, 5}, {1, 5}, {2, 5}, {3, 5}};
static const uint32_t sphere_t[8][3] = {
  {0, 1, 4}, {1, 2, 4}, {2, 3, 4}, {3, 0, 4}, {0, 5, 1}, {1, 5, 2}, {2, 5, 3}, {3, 5, 0}};
static const uint32_t sphere_s[8][3] = {
  {5, 4, 0}, {6, 5, 1}, {7, 6, 2}, {4, 7, 3}, {9, 0, 8}, {10, 1, 9}, {11, 2, 10}, {8, 3, 11}};

/* Cube [-1,1]^3. */
static const double cube_x[8][3] = {
  {-1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}, {-1, 1, 1},
  {1, -1, -1}, {1, 1, -1}, {1, -1, 1}, {1, 1, 1}};
static const uint32_t cube_e[18][2] = {
  {1, 0}, {0, 3}, {3, 1}, {2, 0}, {3, 2}, {5, 7}, {7, 4}, {4, 5}, {4, 6},
  {6, 7}, {2, 6}, {6, 3}, {3, 7}, {5, 1}, {1, 4}, {4, 0}, {1, 7}, {0, 6}};
static const uint32_t cube_t[12][3] = {
  {1, 0, 3}, {3, 0, 2}, {4, 5, 7}, {4, 7, 6}, {3, 2, 6}, {3, 6, 7},
  {4, 0, 1}, {4, 1, 5}, {0, 6, 2}, {4, 6, 0}, {1, 3, 7}, {1, 7, 5}};
static const uint32_t cube_s[12][3] = {
  {1, 2, 0}, {3, 4, 1}, {5, 6, 7}, {9, 8, 6}, {10, 11, 4}, {9, 12, 11},
  {0, 14, 15}, {13, 7, 14}, {10, 3, 17}, {17, 15, 8}, {12, 16, 2}, {5, 13, 16}};

static int
get_macro(int kind, macro_t *m)
{
  switch (kind) {
  case H2B_MESH_SPHERE:
    m->nv = 6; m->ne = 12; m->nt = 8;
    m->x = sphere_x; m->e = sphere_e; m->t = sphere_t; m->s = sphere_s;
    m->project_to_sphere = 1;
    return 0;
  case H2B_MESH_CUBE:
    m->nv = 8; m->ne = 18; m->nt = 12;
    m->x = cube_x; m->e = cube_e; m->t = cube_t; m->s = cube_s;
    m->project_to_sphere = 0;
    return 0;
  default:
    return -1;
  }
}

/* Point with barycentric coordinates (1-a-b, a, b) on macro triangle i, optionally projected. */
static void
macro_point(const macro_t *m, uint32_t i, double a, double b, double out[3])
{
  const double *p0 = m->x[m->t[i][0]], *p1 = m->x[m->t[i][1]], *p2 = m->x[m->t[i][2]];
  int d;
  for (d = 0; d < 3; d++)
    out[d] = p0[d] * (1.0 - a - b) + p1[d] * a + p2[d] * b;
  if (m->project_to_sphere) {
    double r = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    out[0] /= r;
    out[1] /= r;
    out[2] /= r;
  }
}

int
h2b_macro_mesh_size(int kind, uint32_t split, uint32_t *vertices, uint32_t *triangles)
{
  macro_t m;
  if (get_macro(kind, &m) != 0 || split < 1) {
    h2b_set_error("h2b_macro_mesh_size: unknown mesh kind %d or split %u", kind, split);
    return H2B_ERR_ARG;
  }
  *vertices = m.nv + m.ne * (split - 1) + m.nt * (split - 1) * (split - 2) / 2;
  *triangles = m.nt * split * split;
  return H2B_OK;
}

int
h2b_macro_mesh_build(int kind, uint32_t split, double *x, uint32_t *t)
{
  macro_t m;
  uint32_t nv, nt, vcount = 0, tcount = 0, i, j, k, s1 = split + 1;
  uint32_t *vnum, *enum0, *loc;
  char *vdone, *edone;

  if (h2b_macro_mesh_size(kind, split, &nv, &nt) != H2B_OK || get_macro(kind, &m) != 0)
    return H2B_ERR_ARG;

  vnum = (uint32_t *) malloc(sizeof(uint32_t) * m.nv);
  enum0 = (uint32_t *) malloc(sizeof(uint32_t) * m.ne);
  vdone = (char *) calloc(m.nv, 1);
  edone = (char *) calloc(m.ne, 1);
  loc = (uint32_t *) malloc(sizeof(uint32_t) * s1 * s1);
  if (!vnum || !enum0 || !vdone || !edone || !loc) {
    free(vnum); free(enum0); free(vdone); free(edone); free(loc);
    h2b_set_error("h2b_macro_mesh_build: out of host memory");
    return H2B_ERR_NOMEM;
  }

  /* Pass 1: vertices on macro vertices and on macro edges, in order of first appearance. */
  for (i = 0; i < m.nt; i++) {
    for (j = 0; j < 3; j++) {
      uint32_t v = m.t[i][j];
      if (!vdone[v]) {
        static const double bary[3][2] = {{0.0, 0.0}, {1.0, 0.0}, {0.0, 1.0}};
        macro_point(&m, i, bary[j][0], bary[j][1], x + 3 * (size_t) vcount);
        vnum[v] = vcount++;
        vdone[v] = 1;
      }
    }
    for (j = 0; j < 3; j++) {
      uint32_t e = m.s[i][j];
      if (edone[e])
        continue;
      enum0[e] = vcount;
      for (k = 1; k < split; k++) {
        /* fraction along the edge, measured from the edge's first vertex */
        double a = (m.e[e][0] == m.t[i][(j + 1) % 3]) ? (double) k / split
                                                      : (double) (split - k) / split;
        double *p = x + 3 * (size_t) vcount;
        if (j == 0)
          macro_point(&m, i, 1.0 - a, a, p);
        else if (j == 1)
          macro_point(&m, i, 0.0, 1.0 - a, p);
        else
          macro_point(&m, i, a, 0.0, p);
        vcount++;
      }
      edone[e] = 1;
    }
  }

  /* Pass 2: per macro triangle, a local (split+1)^2 grid loc[k + j*(split+1)] of vertex numbers,
   * interior vertices, then the split^2 sub-triangles. */
  for (i = 0; i < m.nt; i++) {
    uint32_t e;
    loc[0] = vnum[m.t[i][0]];
    loc[split] = vnum[m.t[i][1]];
    loc[split * s1] = vnum[m.t[i][2]];

    e = m.s[i][0];  /* edge between local vertices 1 and 2 */
    for (j = 1; j < split; j++) {
      if (m.e[e][0] == m.t[i][1])
        loc[(split - j) + j * s1] = enum0[e] + (j - 1);
      else
        loc[j + (split - j) * s1] = enum0[e] + (j - 1);
    }
    e = m.s[i][1];  /* edge between local vertices 2 and 0 */
    for (j = 1; j < split; j++) {
      if (m.e[e][0] == m.t[i][2])
        loc[(split - j) * s1] = enum0[e] + (j - 1);
      else
        loc[j * s1] = enum0[e] + (j - 1);
    }
    e = m.s[i][2];  /* edge between local vertices 0 and 1 */
    for (j = 1; j < split; j++) {
      if (m.e[e][0] == m.t[i][0])
        loc[j] = enum0[e] + (j - 1);
      else
        loc[split - j] = enum0[e] + (j - 1);
    }

    for (j = 1; j < split; j++) {
      double b = (double) j / split;
      for (k = 1; k < split - j; k++) {
        double a = (double) k / split;
        loc[k + j * s1] = vcount;
        macro_point(&m, i, a, b, x + 3 * (size_t) vcount);
        vcount++;
      }
    }

    for (j = 0; j < split; j++) {
      for (k = 0; k + 1 < split - j; k++) {
        uint32_t *tt = t + 3 * (size_t) tcount;
        tt[0] = loc[k + j * s1];
        tt[1] = loc[(k + 1) + j * s1];
        tt[2] = loc[k + (j + 1) * s1];
        tt += 3;
        tt[0] = loc[(k + 1) + (j + 1) * s1];
        tt[1] = loc[k + (j + 1) * s1];
        tt[2] = loc[(k + 1) + j * s1];
        tcount += 2;
      }
      {
        uint32_t *tt = t + 3 * (size_t) tcount;
        tt[0] = loc[k + j * s1];
        tt[1] = loc[(k + 1) + j * s1];
        tt[2] = loc[k + (j + 1) * s1];
        tcount++;
      }
    }
  }

  free(vnum); free(enum0); free(vdone); free(edone); free(loc);
  if (vcount != nv || tcount != nt) {
    h2b_set_error("h2b_macro_mesh_build: internal count mismatch (%u/%u vertices, %u/%u triangles)",
                  vcount, nv, tcount, nt);
    return H2B_ERR_INTERNAL;
  }
  return H2B_OK;
}

int
h2b_prepare_surface(uint32_t vertices, const double *x, uint32_t triangles, const uint32_t *t,
                    double *n, double *g, double *hminmax)
{
  double hmin = 1e30, hmax = 0.0;
  uint32_t i;

  for (i = 0; i < triangles; i++) {
    const uint32_t *ti = t + 3 * (size_t) i;
    const double *p0, *p1, *p2;
    double dx[3], dy[3], dz[3], nn[3], r, a, b, c, h;
    int d;
    if (ti[0] >= vertices || ti[1] >= vertices || ti[2] >= vertices) {
      h2b_set_error("h2b_prepare_surface: triangle %u references a vertex >= %u", i, vertices);
      return H2B_ERR_ARG;
    }
    p0 = x + 3 * (size_t) ti[0];
    p1 = x + 3 * (size_t) ti[1];
    p2 = x + 3 * (size_t) ti[2];
    for (d = 0; d < 3; d++) {
      dx[d] = p1[d] - p0[d];
      dy[d] = p2[d] - p0[d];
      dz[d] = p2[d] - p1[d];
    }
    nn[0] = dx[1] * dy[2] - dx[2] * dy[1];
    nn[1] = dx[2] * dy[0] - dx[0] * dy[2];
    nn[2] = dx[0] * dy[1] - dx[1] * dy[0];
    r = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
    if (!(r > 0.0)) {
      h2b_set_error("h2b_prepare_surface: triangle %u is degenerate", i);
      return H2B_ERR_ARG;
    }
    g[i] = r;
    n[3 * (size_t) i + 0] = nn[0] / r;
    n[3 * (size_t) i + 1] = nn[1] / r;
    n[3 * (size_t) i + 2] = nn[2] / r;

    a = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    b = sqrt(dy[0] * dy[0] + dy[1] * dy[1] + dy[2] * dy[2]);
    c = sqrt(dz[0] * dz[0] + dz[1] * dz[1] + dz[2] * dz[2]);
    h = 2.0 * fmin(a, fmin(b, c));
    a *= a;
    b *= b;
    c *= c;
    h = sqrt(2 * (a * b + b * c + a * c) - (a * a + b * b + c * c)) / h;
    hmin = fmin(hmin, h);
    hmax = fmax(hmax, h);
  }
  if (hminmax) {
    hminmax[0] = hmin;
    hminmax[1] = hmax;
  }
  return H2B_OK;
}

int
h2b_scale_vertices(uint32_t vertices, double *x, const double scale[3])
{
  uint32_t i;
  for (i = 0; i < vertices; i++) {
    x[3 * (size_t) i + 0] *= scale[0];
    x[3 * (size_t) i + 1] *= scale[1];
    x[3 * (size_t) i + 2] *= scale[2];
  }
  return H2B_OK;
}
