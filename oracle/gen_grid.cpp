// gen_grid.cpp -- TEST INFRASTRUCTURE: writes the new_grid.dat that the
// reference's own airfoil builds read (airfoil/airfoil.cpp:80-129), as a
// stand-alone host program.
//
//     gen_grid I J [scramble seed] out.dat
//
// The reference's mesh generator is MATLAB (airfoil/naca0012.m), absent
// here; the product library restates it (oplus2_matlab_b200/csrc/meshgen.cpp).
// This program links that one host source file directly, so that the timed
// reference run (bench.py --impl reference) and the golden-vector scripts
// can create the reference's input without loading the product's CUDA
// library into their process.
#include <cstdio>
#include <cstdlib>

#include "op2b_mesh.h"

int main(int argc, char **argv) {
  if (argc != 4 && argc != 6) {
    fprintf(stderr, "usage: %s I J [scramble seed] out.dat\n", argv[0]);
    return 2;
  }
  const int I = atoi(argv[1]), J = atoi(argv[2]);
  const int scramble = argc == 6 ? atoi(argv[3]) : 0;
  const unsigned long long seed = argc == 6 ? strtoull(argv[4], nullptr, 10) : 0ull;
  const char *out = argv[argc - 1];
  op2b_mesh m;
  int rc = op2b_mesh_naca0012(I, J, scramble, (uint64_t)seed, &m);
  if (rc != 0) {
    fprintf(stderr, "gen_grid: mesh generation failed (I=%d, J=%d): rc %d\n", I, J, rc);
    return 1;
  }
  rc = op2b_mesh_write(&m, out);
  if (rc == 0)
    printf("%d %d %d %d\n", m.nnode, m.ncell, m.nedge, m.nbedge);
  op2b_mesh_free(&m);
  if (rc != 0) {
    fprintf(stderr, "gen_grid: cannot write %s: rc %d\n", out, rc);
    return 1;
  }
  return 0;
}
