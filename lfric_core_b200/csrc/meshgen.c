/*
 * Synthetic-input generator for the Krylov-solve path: extruded cubed-sphere
 * topology, dofmaps, colouring, perturbed geometry and LMA assembly.
 * See include/lfx_meshgen.h for the conventions and the reference files each
 * part restates. Host code only; compiled with -ffp-contract=off so that the
 * generated matrices do not depend on the compiler's FMA choices.
 */
#include "lfx_meshgen.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SW_ 0
#define SE_ 1
#define NE_ 2
#define NW_ 3
#define W_ 0
#define S_ 1
#define E_ 2
#define N_ 3

/* ------------------------------------------------------------------------- */
/* cubed-sphere topology                                                      */
/* ------------------------------------------------------------------------- */

/* Cell id (1-based) of the i-th cell (1-based) along side s of panel p,
 * listed west->east / south->north (gencube_ps_mod.F90:1943-1973). */
static int32_t edge_cell(int32_t n, int32_t i, int side, int p) {
  int32_t cpp = n * n, base = (p - 1) * cpp;
  switch (side) {
    case W_: return base + n * (i - 1) + 1;
    case S_: return base + (cpp - n) + i;
    case E_: return base + n * i;
    default: return base + i; /* N */
  }
}

/* Panel-edge gluing of gencube_ps_mod.F90:380-545: for panel p and side s,
 * the neighbour is edge_cell(rev ? n+1-i : i, tside, panel_next[p][s]). */
static const int panel_next[7][4] = {{0, 0, 0, 0},
                                     {4, 6, 2, 5},
                                     {1, 6, 3, 5},
                                     {2, 6, 4, 5},
                                     {3, 6, 1, 5},
                                     {1, 2, 3, 4},
                                     {1, 4, 3, 2}};
/* [panel][side] -> {target side, reversed} */
static const int glue[7][4][2] = {
    {{0, 0}, {0, 0}, {0, 0}, {0, 0}},
    /*        W          S          E          N        */
    /* 1 */ {{E_, 0}, {W_, 1}, {W_, 0}, {W_, 0}},
    /* 2 */ {{E_, 0}, {N_, 0}, {W_, 0}, {S_, 0}},
    /* 3 */ {{E_, 0}, {E_, 0}, {W_, 0}, {E_, 1}},
    /* 4 */ {{E_, 0}, {S_, 1}, {W_, 0}, {N_, 1}},
    /* 5 */ {{N_, 0}, {N_, 0}, {N_, 1}, {N_, 1}},
    /* 6 */ {{S_, 1}, {S_, 1}, {S_, 0}, {S_, 0}},
};

#define CN(c, s) cell_next[((c) - 1) * 4 + (s)]
#define VC(c, v) verts_on_cell[((c) - 1) * 4 + (v)]

static void calc_adjacency(int32_t n, int32_t* cell_next) {
  int32_t cpp = n * n, ncells = 6 * cpp;
  for (int32_t c = 1; c <= ncells; ++c) {
    CN(c, W_) = c - 1;
    CN(c, S_) = c + n;
    CN(c, E_) = c + 1;
    CN(c, N_) = c - n;
  }
  /* the reference overwrites N, E, S, W of the panel-edge cells in turn */
  static const int order[4] = {N_, E_, S_, W_};
  for (int p = 1; p <= 6; ++p)
    for (int32_t i = 1; i <= n; ++i)
      for (int o = 0; o < 4; ++o) {
        int s = order[o];
        int32_t c = edge_cell(n, i, s, p);
        int32_t j = glue[p][s][1] ? n + 1 - i : i;
        CN(c, s) = edge_cell(n, j, glue[p][s][0], panel_next[p][s]);
      }
}

/* Vertex numbering, gencube_ps_mod.F90:558-703, before panel re-orientation. */
static void calc_face_to_vert(int32_t n, const int32_t* cell_next,
                              int32_t* verts_on_cell) {
  int32_t cpp = n * n, c, idx, nxf;
  memset(verts_on_cell, 0, sizeof(int32_t) * 4 * 6 * cpp);
  for (c = 1; c <= 4 * cpp; ++c) VC(c, NW_) = c;
  for (c = 1; c <= 4 * cpp; ++c) VC(c, NE_) = VC(CN(c, E_), NW_);
  for (int p = 1; p <= 4; ++p)
    for (c = (p - 1) * cpp + 1; c <= p * cpp - n; ++c) {
      VC(c, SW_) = VC(CN(c, S_), NW_);
      VC(c, SE_) = VC(CN(c, S_), NE_);
    }
  nxf = 4 * cpp + 1;
  for (idx = 0; idx <= n - 2; ++idx)
    for (c = 4 * cpp + idx * n + 1; c <= 4 * cpp + idx * n + n - 1; ++c) {
      VC(c, SE_) = nxf++;
      VC(CN(c, E_), SW_) = VC(c, SE_);
      VC(CN(c, S_), NE_) = VC(c, SE_);
      VC(CN(CN(c, S_), E_), NW_) = VC(c, SE_);
    }
  for (c = 5 * cpp + 1; c <= 6 * cpp; ++c) VC(c, NW_) = nxf++;
  for (c = 5 * cpp + 1; c <= 6 * cpp - n; ++c) VC(c, SW_) = VC(CN(c, S_), NW_);
  for (c = 6 * cpp - n + 1; c <= 6 * cpp; ++c) VC(c, SW_) = nxf++;
  for (c = 3 * cpp - n + 1; c <= 3 * cpp; ++c) {
    VC(c, SW_) = nxf;
    VC(CN(c, W_), SE_) = VC(c, SW_);
    nxf++;
  }
  c = 3 * cpp;
  VC(c, SE_) = nxf;
  VC(CN(c, E_), SW_) = VC(c, SE_);
  for (c = cpp - n + 1; c <= cpp; ++c) {
    VC(c, SW_) = VC(CN(c, S_), SW_);
    VC(c, SE_) = VC(CN(c, S_), NW_);
  }
  for (c = 1; c <= n; ++c) {
    VC(CN(c, N_), NW_) = VC(c, NW_);
    VC(CN(c, N_), SW_) = VC(c, NE_);
  }
  for (c = 2 * cpp + 1; c <= 2 * cpp + n; ++c) {
    VC(CN(c, N_), SE_) = VC(c, NW_);
    VC(CN(c, N_), NE_) = VC(c, NE_);
  }
  for (c = 3 * cpp - n + 1; c <= 3 * cpp; ++c) {
    VC(CN(c, S_), NE_) = VC(c, SW_);
    VC(CN(c, S_), SE_) = VC(c, SE_);
  }
  for (c = 3 * cpp + 1; c <= 3 * cpp + n; ++c) {
    VC(CN(c, N_), NE_) = VC(c, NW_);
    VC(CN(c, N_), NW_) = VC(c, NE_);
  }
  for (idx = 0; idx <= n - 1; ++idx)
    for (c = 5 * cpp + 1 + idx * n; c <= 5 * cpp + 1 + idx * n + n - 2; ++c) {
      VC(c, NE_) = VC(CN(c, E_), NW_);
      VC(c, SE_) = VC(CN(c, E_), SW_);
    }
  for (c = 6 * cpp - n + 1; c <= 6 * cpp; ++c) {
    VC(CN(c, S_), SW_) = VC(c, SE_);
    VC(CN(c, S_), SE_) = VC(c, SW_);
  }
  for (c = 2 * cpp - n + 1; c <= 2 * cpp; ++c) {
    VC(c, SW_) = VC(CN(c, S_), NW_);
    VC(c, SE_) = VC(CN(c, S_), NE_);
  }
  for (c = cpp + 1; c <= cpp + n; ++c) {
    VC(CN(c, N_), SW_) = VC(c, NW_);
    VC(CN(c, N_), SE_) = VC(c, NE_);
  }
}

/* Equiangular gnomonic point of panel-local angles (l1, l2); the reference
 * stores (long, -lat), i.e. the z component is mirrored. */
static void gnomonic(double l1, double l2, double* xs, double* ys, double* zs) {
  double t1 = tan(l1), t2 = tan(l2);
  *xs = 1.0 / sqrt(1.0 + t1 * t1 + t2 * t2);
  *ys = *xs * t1;
  *zs = *xs * t2;
}
static void put(double* xyz, int32_t v, double x, double y, double z) {
  double r = sqrt(x * x + y * y + z * z);
  xyz[(v - 1) * 3 + 0] = x / r;
  xyz[(v - 1) * 3 + 1] = y / r;
  xyz[(v - 1) * 3 + 2] = -z / r;
}

/* gencube_ps_mod.F90:887-1113 */
static void calc_coords(int32_t n, const int32_t* verts_on_cell, double* xyz) {
  int32_t cpp = n * n, x, y, c, v = 1;
  const double pio4 = M_PI / 4.0, dl = 0.5 * M_PI / n;
  double xs, ys, zs;
  for (y = 1; y <= n; ++y)
    for (x = 1; x <= n; ++x, ++v) {
      gnomonic((x - 1) * dl - pio4, (y - 1) * dl - pio4, &xs, &ys, &zs);
      put(xyz, v, xs, ys, zs);
      put(xyz, v + cpp, -ys, xs, zs);
      put(xyz, v + 2 * cpp, -xs, -ys, zs);
      put(xyz, v + 3 * cpp, ys, -xs, zs);
    }
  c = 4 * cpp;
  for (y = 1; y <= n - 1; ++y, c += n)
    for (x = 1; x <= n - 1; ++x) {
      gnomonic(x * dl - pio4, y * dl - pio4, &xs, &ys, &zs);
      put(xyz, VC(c + x, SE_), -ys, zs, -xs);
    }
  c = 5 * cpp + 1;
  for (y = 1; y <= n; ++y)
    for (x = 1; x <= n; ++x, ++c) {
      gnomonic((x - 1) * dl - pio4, (y - 1) * dl - pio4, &xs, &ys, &zs);
      put(xyz, VC(c, NW_), -ys, -zs, xs);
    }
  c = 6 * cpp - n + 1;
  for (x = 1; x <= n; ++x, ++c) {
    gnomonic((x - 1) * dl - pio4, n * dl - pio4, &xs, &ys, &zs);
    put(xyz, VC(c, SW_), -ys, -zs, xs);
  }
  c = 5 * cpp + n;
  for (y = 1; y <= n; ++y, c += n) {
    gnomonic(n * dl - pio4, (y - 1) * dl - pio4, &xs, &ys, &zs);
    put(xyz, VC(c, NE_), -ys, -zs, xs);
  }
  gnomonic(n * dl - pio4, n * dl - pio4, &xs, &ys, &zs);
  put(xyz, 6 * cpp + 2, -ys, -zs, xs);
}

/* orient_lfric (gencube_ps_mod.F90:1561-1602) with PANEL_ROTATIONS (:69):
 * cshift of the 4 entries of verts_on_cell and cell_next on rotated panels. */
static void cshift4(int32_t* a, int shift) {
  int32_t t[4];
  for (int i = 0; i < 4; ++i) t[i] = a[((i + shift) % 4 + 4) % 4];
  memcpy(a, t, sizeof t);
}

int lfx_mg_cubed_sphere(int32_t n, int32_t* cell_next, int32_t* verts_on_cell,
                        double* vert_xyz) {
  static const int rot[6] = {0, 0, 1, 1, -1, 0};
  if (n < 2) return -1;
  int32_t cpp = n * n;
  calc_adjacency(n, cell_next);
  calc_face_to_vert(n, cell_next, verts_on_cell);
  memset(vert_xyz, 0, sizeof(double) * 3 * (6 * cpp + 2));
  calc_coords(n, verts_on_cell, vert_xyz);
  for (int p = 0; p < 6; ++p)
    if (rot[p])
      for (int32_t c = p * cpp; c < (p + 1) * cpp; ++c) {
        cshift4(verts_on_cell + 4 * c, rot[p]);
        cshift4(cell_next + 4 * c, rot[p]);
      }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* colouring                                                                  */
/* ------------------------------------------------------------------------- */

int lfx_mg_test_colours(int32_t ncell, const int32_t* cell_next,
                        const int32_t* colour_map) {
  /* colour_map is indexed by 1-based cell id; id 0 means "no neighbour". */
#define COL(c) ((c) > 0 ? colour_map[(c) - 1] : 0)
  for (int32_t c = 1; c <= ncell; ++c) {
    int32_t col = COL(c);
    if (col == COL(CN(c, N_)) || col == COL(CN(c, S_)) || col == COL(CN(c, E_)) ||
        col == COL(CN(c, W_)))
      return 0;
    int32_t t = CN(c, N_);
    if (t > 0) {
      if (c == CN(t, S_)) {
        if (col == COL(CN(t, E_)) || col == COL(CN(t, W_))) return 0;
      } else if (col == COL(CN(t, N_)) || col == COL(CN(t, S_)))
        return 0;
    }
    t = CN(c, S_);
    if (t > 0) {
      if (c == CN(t, N_)) {
        if (col == COL(CN(t, E_)) || col == COL(CN(t, W_))) return 0;
      } else if (col == COL(CN(t, N_)) || col == COL(CN(t, S_)))
        return 0;
    }
  }
  return 1;
}

/* set_colours_generic (mesh_colouring_mod.F90:520-650): greedy smallest free. */
static int colour_generic(int32_t ncell, const int32_t* cell_next,
                          int32_t* colour_map) {
  enum { MAXCOLS = 50 };
  int ncol = 0;
  memset(colour_map, 0, sizeof(int32_t) * ncell);
  for (int32_t c = 1; c <= ncell; ++c) {
    int used[MAXCOLS + 1] = {0};
    int32_t t = CN(c, N_);
    if (t > 0) {
      used[COL(t)] = 1;
      if (c == CN(t, S_)) {
        used[COL(CN(t, E_))] = 1;
        used[COL(CN(t, W_))] = 1;
      } else {
        used[COL(CN(t, N_))] = 1;
        used[COL(CN(t, S_))] = 1;
      }
    }
    t = CN(c, E_);
    if (t > 0) used[COL(t)] = 1;
    t = CN(c, W_);
    if (t > 0) used[COL(t)] = 1;
    t = CN(c, S_);
    if (t > 0) {
      used[COL(t)] = 1;
      if (c == CN(t, N_)) {
        used[COL(CN(t, E_))] = 1;
        used[COL(CN(t, W_))] = 1;
      } else {
        used[COL(CN(t, N_))] = 1;
        used[COL(CN(t, S_))] = 1;
      }
    }
    int free_c = 0;
    for (int i = 1; i <= MAXCOLS; ++i)
      if (!used[i]) {
        free_c = i;
        break;
      }
    if (!free_c) return -1;
    colour_map[c - 1] = free_c;
    if (free_c > ncol) ncol = free_c;
  }
  return ncol;
}

int lfx_mg_colour_cubed_sphere(int32_t n, const int32_t* cell_next,
                               int32_t* colour_map) {
  /* 2x2 panel patterns (column, row) per panel, mesh_colouring_mod.F90:241-268.
   * Fortran reshape((/a,b,c,d/),(/2,2/)) gives (1,1)=a,(2,1)=b,(1,2)=c,(2,2)=d. */
  static const int even[6][4] = {{1, 2, 3, 4}, {3, 2, 1, 4}, {3, 4, 1, 2},
                                 {1, 4, 3, 2}, {3, 2, 4, 1}, {2, 3, 1, 4}};
  static const int odd[6][4] = {{1, 2, 3, 4}, {4, 1, 2, 3}, {1, 2, 3, 4},
                                {4, 1, 2, 3}, {3, 2, 4, 1}, {3, 2, 4, 1}};
  int32_t cpp = n * n, ncell = 6 * cpp;
  for (int32_t gid = 1; gid <= ncell; ++gid) {
    int32_t panel = (gid - 1) / cpp + 1;
    int32_t g = gid - cpp * (panel - 1);
    int column = 2 - ((g % n) % 2);
    int row = ((g - 1) / n) % 2 + 1;
    const int* t = (n % 2 == 0) ? even[panel - 1] : odd[panel - 1];
    colour_map[gid - 1] = t[(column - 1) + 2 * (row - 1)];
  }
  if (lfx_mg_test_colours(ncell, cell_next, colour_map)) return 4;
  int nc = colour_generic(ncell, cell_next, colour_map);
  if (nc < 0 || !lfx_mg_test_colours(ncell, cell_next, colour_map)) return -1;
  return nc;
}

/* ------------------------------------------------------------------------- */
/* dofmaps                                                                    */
/* ------------------------------------------------------------------------- */

/* Side of cell t that faces cell c (or -1). */
static int back_side(const int32_t* cell_next, int32_t t, int32_t c) {
  for (int s = 0; s < 4; ++s)
    if (CN(t, s) == c) return s;
  return -1;
}

int64_t lfx_mg_dofmap(int32_t space, int32_t ncell, int32_t nlayers,
                      const int32_t* cell_next, const int32_t* verts_on_cell,
                      int32_t* map) {
  int64_t id = 1;
  if (space == LFX_MG_W3) {
    for (int32_t c = 0; c < ncell; ++c, id += nlayers) map[c] = (int32_t)id;
    return id - 1;
  }
  if (space == LFX_MG_W0) {
    int32_t nv = 0;
    for (int32_t i = 0; i < 4 * ncell; ++i)
      if (verts_on_cell[i] > nv) nv = verts_on_cell[i];
    int32_t* base = (int32_t*)calloc((size_t)nv + 1, sizeof(int32_t));
    if (!base) return -1;
    for (int32_t c = 1; c <= ncell; ++c)
      for (int v = 0; v < 4; ++v) {
        int32_t vid = VC(c, v);
        if (!base[vid]) {
          base[vid] = (int32_t)id;
          id += nlayers + 1;
        }
        map[(c - 1) * 8 + v] = base[vid];
        map[(c - 1) * 8 + v + 4] = base[vid] + 1;
      }
    free(base);
    return id - 1;
  }
  if (space == LFX_MG_W2) {
    /* horizontal faces W,S,E,N then the bottom/top vertical-face column */
    int32_t* fbase = (int32_t*)calloc((size_t)ncell * 4, sizeof(int32_t));
    if (!fbase) return -1;
    for (int32_t c = 1; c <= ncell; ++c) {
      for (int s = 0; s < 4; ++s) {
        int32_t t = CN(c, s);
        int32_t* slot = &fbase[(c - 1) * 4 + s];
        if (!*slot) {
          *slot = (int32_t)id;
          id += nlayers;
          int bs = back_side(cell_next, t, c);
          if (bs < 0) {
            free(fbase);
            return -1;
          }
          fbase[(t - 1) * 4 + bs] = *slot;
        }
        map[(c - 1) * 6 + s] = *slot;
      }
      map[(c - 1) * 6 + 4] = (int32_t)id;
      map[(c - 1) * 6 + 5] = (int32_t)id + 1;
      id += nlayers + 1;
    }
    free(fbase);
    return id - 1;
  }
  return -1;
}

/* ------------------------------------------------------------------------- */
/* seeded samples and geometry                                                */
/* ------------------------------------------------------------------------- */

static uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
/* uniform in [0,1) from (seed, counter) */
static double u01(uint64_t seed, uint64_t i) {
  uint64_t h = splitmix64(seed * 0x632be59bd9b4e019ULL ^ splitmix64(i));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

void lfx_mg_uniform(uint64_t seed, int64_t n, double lo, double hi, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * u01(seed, (uint64_t)i);
}

void lfx_mg_normal(uint64_t seed, int64_t n, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i += 2) {
    double u1 = 1.0 - u01(seed, (uint64_t)i), u2 = u01(seed, (uint64_t)i + 1);
    double r = sqrt(-2.0 * log(u1)), th = 2.0 * M_PI * u2;
    out[i] = r * cos(th);
    if (i + 1 < n) out[i + 1] = r * sin(th);
  }
}

int lfx_mg_geometry(int32_t n, int32_t nlayers, const double* vert_xyz,
                    uint64_t seed, double perturb, double* xyz3d) {
  int64_t nv = 6LL * n * n + 2;
  double h0 = 0.5 * M_PI / n;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < nv; ++v)
    for (int32_t l = 0; l <= nlayers; ++l) {
      double r = 1.0 + l * h0, h = r * h0;
      int64_t p = v * (nlayers + 1) + l;
      for (int a = 0; a < 3; ++a) {
        double u = u01(seed, (uint64_t)(p * 3 + a));
        xyz3d[p * 3 + a] = r * vert_xyz[v * 3 + a] + perturb * h * (2.0 * u - 1.0);
      }
    }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* LMA assembly                                                               */
/* ------------------------------------------------------------------------- */

/* reference-cube vertex coordinates, SWB..NWT (reference_element_mod.F90:1244) */
static const double rv[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

static void gauss3(double* x, double* w) {
  double d = sqrt(15.0) / 10.0;
  x[0] = 0.5 - d;
  x[1] = 0.5;
  x[2] = 0.5 + d;
  w[0] = 5.0 / 18.0;
  w[1] = 8.0 / 18.0;
  w[2] = 5.0 / 18.0;
}

/* trilinear basis and reference gradients at xi */
static void q1(const double* xi, double* phi, double (*dphi)[3]) {
  for (int v = 0; v < 8; ++v) {
    double f[3], g[3];
    for (int a = 0; a < 3; ++a) {
      f[a] = rv[v][a] > 0.5 ? xi[a] : 1.0 - xi[a];
      g[a] = rv[v][a] > 0.5 ? 1.0 : -1.0;
    }
    phi[v] = f[0] * f[1] * f[2];
    dphi[v][0] = g[0] * f[1] * f[2];
    dphi[v][1] = f[0] * g[1] * f[2];
    dphi[v][2] = f[0] * f[1] * g[2];
  }
}

/* corner positions of cell c (0-based), layer k, reference vertex order */
static void cell_corners(int32_t c, int32_t k, int32_t nlayers,
                         const int32_t* verts_on_cell, const double* xyz3d,
                         double X[8][3]) {
  for (int v = 0; v < 8; ++v) {
    int64_t vid = verts_on_cell[c * 4 + (v & 3)] - 1;
    int64_t p = vid * (nlayers + 1) + k + (v >> 2);
    for (int a = 0; a < 3; ++a) X[v][a] = xyz3d[p * 3 + a];
  }
}

static double jacobian(double X[8][3], double (*dphi)[3], double J[3][3]) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = 0.0;
      for (int v = 0; v < 8; ++v) s += X[v][a] * dphi[v][b];
      J[a][b] = s;
    }
  return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

#define LMA(arr, ik, i, j, ndf_to, ncell3d) \
  (arr)[(int64_t)(ik) + (int64_t)(ncell3d) * ((i) + (int64_t)(ndf_to) * (j))]

int lfx_mg_lma_w0(int32_t ncell, int32_t nlayers, const int32_t* verts_on_cell,
                  const double* xyz3d, double nu, double* lma) {
  double gx[3], gw[3];
  gauss3(gx, gw);
  int64_t ncell3d = (int64_t)ncell * nlayers;
#pragma omp parallel for schedule(static)
  for (int64_t ik = 0; ik < ncell3d; ++ik) {
    int32_t c = (int32_t)(ik / nlayers), k = (int32_t)(ik % nlayers);
    double X[8][3], A[8][8] = {{0}};
    cell_corners(c, k, nlayers, verts_on_cell, xyz3d, X);
    for (int q = 0; q < 27; ++q) {
      double xi[3] = {gx[q % 3], gx[(q / 3) % 3], gx[q / 9]};
      double wq = gw[q % 3] * gw[(q / 3) % 3] * gw[q / 9];
      double phi[8], dphi[8][3], J[3][3], G[3][3];
      q1(xi, phi, dphi);
      double dj = jacobian(X, dphi, J), adj = fabs(dj);
      /* G = (J^T J)^{-1} via the inverse of J */
      double Ji[3][3];
      Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / dj;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / dj;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / dj;
      Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / dj;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / dj;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / dj;
      Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / dj;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / dj;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / dj;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          G[a][b] = Ji[a][0] * Ji[b][0] + Ji[a][1] * Ji[b][1] + Ji[a][2] * Ji[b][2];
      /* the upper triangle; the lower one is its mirror image, so the
       * local matrix is symmetric bit for bit */
      for (int i = 0; i < 8; ++i)
        for (int j = i; j < 8; ++j) {
          double kij = 0.0;
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) kij += dphi[i][a] * G[a][b] * dphi[j][b];
          A[i][j] += wq * adj * (phi[i] * phi[j] + nu * kij);
        }
    }
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) LMA(lma, ik, i, j, 8, ncell3d) = i <= j ? A[i][j] : A[j][i];
  }
  return 0;
}

/* RT0 reference basis, faces W,S,E,N,B,T, each with unit outward flux on its
 * own face and divergence +1 on the unit cube. */
static void rt0(const double* xi, double v[6][3]) {
  memset(v, 0, sizeof(double) * 18);
  v[0][0] = xi[0] - 1.0; /* W */
  v[1][1] = xi[1] - 1.0; /* S */
  v[2][0] = xi[0];       /* E */
  v[3][1] = xi[1];       /* N */
  v[4][2] = xi[2] - 1.0; /* B */
  v[5][2] = xi[2];       /* T */
}

int lfx_mg_lma_w2(int32_t ncell, int32_t nlayers, const int32_t* cell_next,
                  const int32_t* verts_on_cell, const double* xyz3d, double tau,
                  double* m2, double* div, double* a) {
  double gx[3], gw[3];
  gauss3(gx, gw);
  int64_t ncell3d = (int64_t)ncell * nlayers;
#pragma omp parallel for schedule(static)
  for (int64_t ik = 0; ik < ncell3d; ++ik) {
    int32_t c = (int32_t)(ik / nlayers), k = (int32_t)(ik % nlayers);
    /* one global normal per face: outward from the lower-numbered cell on
     * horizontal faces, upward on vertical faces */
    double sg[6];
    for (int s = 0; s < 4; ++s) sg[s] = (c + 1 < cell_next[c * 4 + s]) ? 1.0 : -1.0;
    sg[4] = -1.0;
    sg[5] = 1.0;
    double X[8][3], M[6][6] = {{0}}, D[6];
    cell_corners(c, k, nlayers, verts_on_cell, xyz3d, X);
    for (int q = 0; q < 27; ++q) {
      double xi[3] = {gx[q % 3], gx[(q / 3) % 3], gx[q / 9]};
      double wq = gw[q % 3] * gw[(q / 3) % 3] * gw[q / 9];
      double phi[8], dphi[8][3], J[3][3], v[6][3], Jv[6][3];
      q1(xi, phi, dphi);
      double adj = fabs(jacobian(X, dphi, J));
      rt0(xi, v);
      for (int i = 0; i < 6; ++i)
        for (int r = 0; r < 3; ++r)
          Jv[i][r] = J[r][0] * v[i][0] + J[r][1] * v[i][1] + J[r][2] * v[i][2];
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
          M[i][j] += wq * sg[i] * sg[j] *
                     (Jv[i][0] * Jv[j][0] + Jv[i][1] * Jv[j][1] + Jv[i][2] * Jv[j][2]) /
                     adj;
    }
    for (int i = 0; i < 6; ++i) D[i] = sg[i]; /* int sigma * div(v_i), sigma = 1 */
    for (int i = 0; i < 6; ++i) {
      if (div) LMA(div, ik, 0, i, 1, ncell3d) = D[i];
      for (int j = 0; j < 6; ++j) {
        if (m2) LMA(m2, ik, i, j, 6, ncell3d) = M[i][j];
        if (a) LMA(a, ik, i, j, 6, ncell3d) = M[i][j] + tau * D[i] * D[j];
      }
    }
  }
  return 0;
}
