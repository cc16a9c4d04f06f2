/*
 * op2b_mesh.h -- airfoil mesh generation and the new_grid.dat text format.
 *
 * The reference ships no mesh: its airfoil apps read "new_grid.dat", which the
 * MATLAB script airfoil/naca0012.m writes (new-style section, naca0012.m:203-351;
 * reader airfoil/airfoil.cpp:80-129).  MATLAB is not available, so this library
 * restates that generator in C++ (oplus2_matlab_b200/csrc/meshgen.cpp):
 *   - NACA0012 upper surface, complex square-root transform (naca0012.m:8-29)
 *   - not-a-knot cubic spline of the transformed surface (naca0012.m:45-49)
 *   - C-type grid of 3I x J cells mapped back by z^2 (naca0012.m:51-63)
 *   - new-style edge / boundary-edge numbering and orientation (naca0012.m:203-308)
 *
 * Node coordinates are produced exactly as the reference app sees them: each
 * value is printed with "%f" (naca0012.m:334) and parsed back with strtod (x64)
 * and strtof (x32), so a mesh built in memory equals one read from the file.
 *
 * An optional seeded permutation of the cell, node, edge and bedge numbering
 * (splitmix64 + Fisher-Yates) gives the "scrambled" meshes.
 */
#ifndef OP2B_MESH_H
#define OP2B_MESH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int     nnode, ncell, nedge, nbedge;
  int    *cell;    /* 4*ncell  cell -> nodes               (pcell)   */
  int    *edge;    /* 2*nedge  edge -> nodes               (pedge)   */
  int    *ecell;   /* 2*nedge  edge -> cells               (pecell)  */
  int    *bedge;   /* 2*nbedge boundary edge -> nodes      (pbedge)  */
  int    *becell;  /* nbedge   boundary edge -> cell       (pbecell) */
  int    *bound;   /* nbedge   1 = wall, 2 = far field               */
  double *x64;     /* 2*nnode  coordinates parsed as double          */
  float  *x32;     /* 2*nnode  coordinates parsed as float           */
} op2b_mesh;

/* Build the I x J NACA0012 C-mesh (3I*J cells).  scramble != 0 permutes all
 * four numberings with the splitmix64 stream seeded by `seed`.  Returns 0 on
 * success, nonzero on bad sizes or allocation failure.  Arrays are malloc'd. */
int  op2b_mesh_naca0012(int I, int J, int scramble, uint64_t seed, op2b_mesh *out);
void op2b_mesh_free(op2b_mesh *m);

/* Write / read the new_grid.dat text format (naca0012.m:328-351). */
int  op2b_mesh_write(const op2b_mesh *m, const char *path);
int  op2b_mesh_read(const char *path, op2b_mesh *out);

/* Binary mesh files: the arrays of an op2b_mesh with a header and a hash of
 * the payload (reading a damaged file fails).  op2b_mesh_read_cached reads
 * text_path through a binary cache: when cache_path holds a valid cache of
 * the same text file (same size and modification time) it is read instead
 * of parsing the text; otherwise the text is parsed and the cache written.
 * Returns 0 on success. */
int  op2b_mesh_write_bin(const op2b_mesh *m, const char *path);
int  op2b_mesh_read_bin(const char *path, op2b_mesh *out);
int  op2b_mesh_read_cached(const char *text_path, const char *cache_path, op2b_mesh *out);

/* The jac1 / jac2 test problem (jac1/jac.cpp:65-117): an (NN-1)^2 interior
 * grid stored unstructured, one self edge (A = -1) per node and one edge per
 * interior 4-neighbour (A = 0.25), boundary neighbours adding 0.25 to r.
 * Edges are numbered in the reference's generation order (i outer, j inner).
 * Caller allocates: pp[2*nedge], A[astride*nedge] (doubles for jac2 are
 * written by op2b_mesh_jac2), r[rstride*nnode].  Returns nedge. */
int  op2b_jac_sizes(int NN, int *nnode, int *nedge);
int  op2b_mesh_jac1(int NN, int *pp, float *A, float *r);
int  op2b_mesh_jac2(int NN, int *pp, double *A, float *r);

/* splitmix64 step, exported so every caller draws from the same stream. */
uint64_t op2b_splitmix64(uint64_t *state);

#ifdef __cplusplus
}
#endif

#endif
