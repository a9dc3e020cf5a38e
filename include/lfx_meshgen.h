/*
 * lfx_meshgen.h -- host-side generator of the synthetic inputs a Krylov solve
 * consumes: extruded cubed-sphere topology, column-contiguous dofmaps, the
 * 4-colouring, perturbed trilinear geometry and per-cell local matrices (LMA).
 *
 * In LFRic these arrays come from the mesh generator, the partitioner and the
 * FEM set-up kernels; they are inputs to the solve, not part of it. This
 * generator restates the pieces that fix their layout and numbering:
 *   - cubed-sphere adjacency / vertex numbering / coordinates:
 *       mesh_tools/source/support/gencube_ps_mod.F90:336-546 (calc_adjacency),
 *       :558-703 (calc_face_to_vert), :887-1113 (calc_coords),
 *       :1561-1602 (orient_lfric, PANEL_ROTATIONS :69)
 *   - 4-colouring: infrastructure/source/mesh/mesh_colouring_mod.F90:151-328
 *       (set_colours_cubed_sphere), :520-650 (set_colours_generic),
 *       :765-837 (test_set_colours)
 *   - dof numbering: infrastructure/source/function_space/
 *       function_space_constructor_helper_functions_mod.F90:1715-2317
 *   - LMA assembly by 3x3x3 Gauss quadrature: the W0 / W2 mass and divergence
 *       kernels under components/science/source/kernel/fem/.
 *
 * Conventions (all arrays row-major C, ids 1-based as in the reference):
 *   cell_next[c*4 + s]       s = 0..3 for W,S,E,N  (reference_element_mod W..N)
 *   verts_on_cell[c*4 + v]   v = 0..3 for SWB,SEB,NEB,NWB
 *   map[c*ndf + df]          first (layer-0) dof id of local dof df in column c
 *   local matrices           Fortran order (ncell_3d, ndf_to, ndf_from),
 *                            ik = c*nlayers + k fastest.
 */
#ifndef LFX_MESHGEN_H
#define LFX_MESHGEN_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum lfx_mg_space { LFX_MG_W0 = 0, LFX_MG_W2 = 2, LFX_MG_W3 = 3 };

/* Cubed sphere with n cells per panel edge: 6 n^2 cells, 6 n^2 + 2 vertices.
 * vert_xyz receives unit-sphere positions (3 per vertex). Returns 0 on success. */
int lfx_mg_cubed_sphere(int32_t n, int32_t* cell_next, int32_t* verts_on_cell,
                        double* vert_xyz);

/* Colour map (1-based colours) for the cubed sphere; falls back to the greedy
 * generic colouring when the panel pattern fails the conflict test.
 * Returns the number of colours, or -1 if no valid colouring was found. */
int lfx_mg_colour_cubed_sphere(int32_t n, const int32_t* cell_next,
                               int32_t* colour_map);

/* Conflict test of a colouring (restates test_set_colours): 1 = valid. */
int lfx_mg_test_colours(int32_t ncell, const int32_t* cell_next,
                        const int32_t* colour_map);

/* Column-contiguous dofmap of space W0 (ndf 8), W2 (ndf 6) or W3 (ndf 1).
 * Returns undf (number of unique dofs) or -1 on error. */
int64_t lfx_mg_dofmap(int32_t space, int32_t ncell, int32_t nlayers,
                      const int32_t* cell_next, const int32_t* verts_on_cell,
                      int32_t* map);

/* Extruded, perturbed vertex positions: xyz3d[(v*(nlayers+1) + l)*3 + a].
 * Level l sits at radius 1 + l*h0 with h0 = (pi/2)/n; every coordinate of
 * every vertex moves by U(-perturb, perturb) * h_l, h_l = (1+l*h0)*h0. */
int lfx_mg_geometry(int32_t n, int32_t nlayers, const double* vert_xyz,
                    uint64_t seed, double perturb, double* xyz3d);

/* W0 (Q1 nodal) local matrices A = M + nu*K, Fortran (ncell_3d, 8, 8). */
int lfx_mg_lma_w0(int32_t ncell, int32_t nlayers, const int32_t* verts_on_cell,
                  const double* xyz3d, double nu, double* lma);

/* W2 (RT0) mass M2 (ncell_3d,6,6), W3<-W2 divergence D (ncell_3d,1,6) and the
 * summed operator A = M2 + tau*D^T D (ncell_3d,6,6). Any output may be NULL. */
int lfx_mg_lma_w2(int32_t ncell, int32_t nlayers, const int32_t* cell_next,
                  const int32_t* verts_on_cell, const double* xyz3d, double tau,
                  double* m2, double* div, double* a);

/* Counter-based seeded samples (identical for any thread count). */
void lfx_mg_uniform(uint64_t seed, int64_t n, double lo, double hi, double* out);
void lfx_mg_normal(uint64_t seed, int64_t n, double* out);

#ifdef __cplusplus
}
#endif
#endif
