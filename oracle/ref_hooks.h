/*
 * ref_hooks.h -- force-included (-include) into the reference apps that
 * oracle/Makefile compiles into oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 *
 * The recipe edits the reference app sources only by sed, and only in three
 * places: the iteration count (airfoil/airfoil.cpp:195, jac1/jac.cpp:63-64),
 * the rms print interval and the precision of the printed history.  Those
 * edits call op2ref_env_int() so one binary serves every test size.
 */
#ifndef OP2REF_HOOKS_H
#define OP2REF_HOOKS_H
#include <stdlib.h>

static inline int op2ref_env_int(const char *name, int def) {
  const char *s = getenv(name);
  return (s && *s) ? atoi(s) : def;
}

#endif
