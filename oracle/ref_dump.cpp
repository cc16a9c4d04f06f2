// ref_dump.cpp -- linked into the reference apps built by oracle/Makefile.
// TEST INFRASTRUCTURE ONLY: never part of the product path.
//
// The reference apps end with op_timing_output() (airfoil/airfoil.cpp:256,
// jac1/jac.cpp:196).  The recipe compiles common/op_lib_core.c with
// -Dop_timing_output=op2ref_timing_output_core, and this file supplies the
// real op_timing_output(): when OP2REF_DUMP names a directory, it writes every
// declared dataset (OP_dat_list, common/op_lib_core.c:53) there as raw bytes,
// <name>.bin, so tests can compare the final fields bit for bit.  It then
// prints the reference's own timing table.

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "op_lib_core.h"

extern "C" void op2ref_timing_output_core();
extern int OP_dat_index;
extern op_dat *OP_dat_list;

extern "C" void op_timing_output() {
  const char *dir = getenv("OP2REF_DUMP");
  if (dir && *dir) {
    char path[4096];
    for (int i = 0; i < OP_dat_index; i++) {
      op_dat d = OP_dat_list[i];
      snprintf(path, sizeof path, "%s/%s.bin", dir, d->name);
      FILE *fp = fopen(path, "wb");
      if (!fp) { printf("op2ref: cannot write %s\n", path); exit(1); }
      fwrite(d->data, (size_t)d->size, (size_t)d->set->size, fp);
      fclose(fp);
    }
  }
  op2ref_timing_output_core();
}
