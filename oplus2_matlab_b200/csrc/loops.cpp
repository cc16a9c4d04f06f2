// loops.cpp -- op_par_loop entry points and their dispatch.
//
// The reference generates one host stub per loop (op2.m; e.g.
// airfoil/res_calc_kernel.cu:158-245).  Here every op_par_loop_<name> entry
// point, and the generic op2b_par_loop, check their arguments the way
// op_arg_check does (common/op_lib_core.c:266-305) and then match the
// argument signature (access, dims, types, direct or indirect) against the
// loops this library implements on the device.  A call that matches none is
// an error, never a host fallback.

#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <set>

#include "loops.h"

namespace op2b {

int effective_strategy(char const *loop_name) {
  (void)loop_name;
  int s = rt().strategy;
  return s == OP2B_STRATEGY_COLOURED ? OP2B_STRATEGY_COLOURED : OP2B_STRATEGY_GATHER;
}

double compulsory_bytes(op_set set, int nargs, const op_arg *args) {
  // every distinct map and dataset once (no allocation: this runs per call)
  double bytes = 0;
  for (int m = 0; m < nargs; m++) {
    const op_arg &a = args[m];
    if (a.argtype != OP_ARG_DAT || !a.dat) continue;
    bool map_new = a.map != nullptr, dat_new = true;
    for (int j = 0; j < m; j++) {
      if (args[j].argtype != OP_ARG_DAT) continue;
      if (a.map && args[j].map == a.map) map_new = false;
      if (args[j].dat == a.dat) dat_new = false;
    }
    if (map_new) bytes += 4.0 * a.map->dim * (double)set->size;
    if (dat_new) {
      double fac = (a.acc == OP_READ || a.acc == OP_WRITE) ? 1.0 : 2.0;
      bytes += fac * a.dat->size * (double)a.dat->set->size;
    }
  }
  return bytes;
}

}  // namespace op2b

using namespace op2b;

namespace {

bool dat_arg(const op_arg &a, int dim, op_access acc, bool indirect, const char *type = nullptr) {
  if (a.argtype != OP_ARG_DAT || !a.dat || a.dim != dim || a.acc != acc) return false;
  if (indirect != (a.map != nullptr)) return false;
  if (type && strcmp(a.dat->type, type) != 0) return false;
  return true;
}

bool gbl_arg(const op_arg &a, int dim, op_access acc, const char *type) {
  return a.argtype == OP_ARG_GBL && a.dim == dim && a.acc == acc && a.type &&
         strcmp(a.type, type) == 0 && a.data != nullptr;
}

bool real_type(const op_arg &a, const char *&t) {
  if (!a.dat) return false;
  if (strcmp(a.dat->type, "float") == 0 || strcmp(a.dat->type, "double") == 0) {
    if (!t) t = a.dat->type;
    return strcmp(a.dat->type, t) == 0;
  }
  return false;
}

bool same_types(const op_arg *args, std::initializer_list<int> which) {
  const char *t = nullptr;
  for (int i : which)
    if (!real_type(args[i], t)) return false;
  return true;
}

// airfoil/airfoil_op.cpp:245-292 argument lists
bool is_save_soln(int n, const op_arg *a) {
  return n == 2 && dat_arg(a[0], 4, OP_READ, false) && dat_arg(a[1], 4, OP_WRITE, false) &&
         same_types(a, {0, 1});
}
bool is_adt_calc(int n, const op_arg *a) {
  return n == 6 && dat_arg(a[0], 2, OP_READ, true) && dat_arg(a[1], 2, OP_READ, true) &&
         dat_arg(a[2], 2, OP_READ, true) && dat_arg(a[3], 2, OP_READ, true) &&
         dat_arg(a[4], 4, OP_READ, false) && dat_arg(a[5], 1, OP_WRITE, false) &&
         same_types(a, {0, 1, 2, 3, 4, 5});
}
bool is_res_calc(int n, const op_arg *a) {
  return n == 8 && dat_arg(a[0], 2, OP_READ, true) && dat_arg(a[1], 2, OP_READ, true) &&
         dat_arg(a[2], 4, OP_READ, true) && dat_arg(a[3], 4, OP_READ, true) &&
         dat_arg(a[4], 1, OP_READ, true) && dat_arg(a[5], 1, OP_READ, true) &&
         dat_arg(a[6], 4, OP_INC, true) && dat_arg(a[7], 4, OP_INC, true) &&
         a[6].dat == a[7].dat && a[0].dat == a[1].dat && a[2].dat == a[3].dat &&
         a[4].dat == a[5].dat && same_types(a, {0, 1, 2, 3, 4, 5, 6, 7});
}
bool is_bres_calc(int n, const op_arg *a) {
  return n == 6 && dat_arg(a[0], 2, OP_READ, true) && dat_arg(a[1], 2, OP_READ, true) &&
         dat_arg(a[2], 4, OP_READ, true) && dat_arg(a[3], 1, OP_READ, true) &&
         dat_arg(a[4], 4, OP_INC, true) && dat_arg(a[5], 1, OP_READ, false, "int") &&
         a[0].dat == a[1].dat && same_types(a, {0, 1, 2, 3, 4});
}
bool is_airfoil_update(int n, const op_arg *a) {
  if (n != 5 || !dat_arg(a[0], 4, OP_READ, false) || !dat_arg(a[1], 4, OP_WRITE, false) ||
      !dat_arg(a[2], 4, OP_RW, false) || !dat_arg(a[3], 1, OP_READ, false) ||
      !same_types(a, {0, 1, 2, 3}))
    return false;
  return gbl_arg(a[4], 1, OP_INC, a[0].dat->type);
}
// jac1/jac_op.cpp:168-181, jac2/jac_op.cpp likewise
int jac_res_variant(int n, const op_arg *a) {
  if (n != 4 || !gbl_arg(a[3], 1, OP_READ, "float")) return 0;
  if (dat_arg(a[0], 1, OP_READ, false, "float") && dat_arg(a[1], 1, OP_READ, true, "float") &&
      dat_arg(a[2], 1, OP_INC, true, "float"))
    return 1;
  if (dat_arg(a[0], 3, OP_READ, false, "double") && dat_arg(a[1], 2, OP_READ, true, "float") &&
      dat_arg(a[2], 3, OP_INC, true, "float"))
    return 2;
  return 0;
}
int jac_update_variant(int n, const op_arg *a) {
  if (n != 5 || !gbl_arg(a[3], 1, OP_INC, "float") || !gbl_arg(a[4], 1, OP_MAX, "float"))
    return 0;
  if (dat_arg(a[0], 1, OP_READ, false, "float") && dat_arg(a[1], 1, OP_RW, false, "float") &&
      dat_arg(a[2], 1, OP_INC, false, "float"))
    return 1;
  if (dat_arg(a[0], 2, OP_READ, false, "float") && dat_arg(a[1], 3, OP_RW, false, "float") &&
      dat_arg(a[2], 2, OP_INC, false, "float"))
    return 2;
  return 0;
}

enum Kind { K_NONE, K_SAVE, K_ADT, K_RES, K_BRES, K_AUPDATE, K_JRES, K_JUPDATE };

Kind classify(int nargs, const op_arg *args, int *variant) {
  *variant = 0;
  if (is_res_calc(nargs, args)) return K_RES;
  if (is_adt_calc(nargs, args)) return K_ADT;
  if (is_bres_calc(nargs, args)) return K_BRES;
  if (is_save_soln(nargs, args)) return K_SAVE;
  if (is_airfoil_update(nargs, args)) return K_AUPDATE;
  if ((*variant = jac_res_variant(nargs, args))) return K_JRES;
  if ((*variant = jac_update_variant(nargs, args))) return K_JUPDATE;
  return K_NONE;
}

void run_kind(Kind k, int variant, char const *name, op_set set, const op_arg *args) {
  switch (k) {
    case K_RES: return run_res_calc(name, set, args);
    case K_ADT: return run_adt_calc(name, set, args);
    case K_BRES: return run_bres_calc(name, set, args);
    case K_SAVE: return run_save_soln(name, set, args);
    case K_AUPDATE: return run_airfoil_update(name, set, args);
    case K_JRES: return run_jac_res(name, set, args, variant);
    case K_JUPDATE: return run_jac_update(name, set, args, variant);
    default: return;
  }
}

// The loops held back in case the next call can be fused with them: one of
// save_soln, update, res_calc; res_calc+bres_calc; res_calc+bres_calc+update;
// res_calc+bres_calc+update+save_soln.
struct Held {
  Kind kind = K_NONE;
  std::string name;
  op_set set = nullptr;
  std::vector<op_arg> args;
  bool flux_done = false;  // res_calc: its flux pass already ran (run ahead)
  bool res_zero = false;   // res_calc: res held +0.0 everywhere at the call
};
std::vector<Held> g_chain;

bool dat_in(op_dat d, std::initializer_list<op_dat> ds) {
  for (op_dat x : ds)
    if (x == d) return true;
  return false;
}

// update(qold, q W, res RW, adt) then adt_calc(x via map, q' = q, adt' = adt)
bool adt_follows_update(const op_arg *u, op_set uset, op_set set, const op_arg *a) {
  op_dat q = u[1].dat, res = u[2].dat, adt = u[3].dat;
  if (set != uset || a[4].dat != q || a[5].dat != adt) return false;
  for (int i = 0; i < 4; i++)
    if (dat_in(a[i].dat, {q, res, adt})) return false;
  return true;
}

// res_calc(x, q, adt -> res INC), bres_calc(x, q, adt, bound -> res INC)
bool bres_follows_res(const op_arg *r, const op_arg *b) {
  op_dat res = r[6].dat;
  if (b[4].dat != res) return false;
  for (int i : {0, 1, 2, 3, 5})
    if (b[i].dat == res) return false;
  return true;
}

// update(qold, q, res, adt) on the cells res_calc/bres_calc increment: it
// reads their result only at its own cell and writes nothing they read
// (their reads all finish in the flux pass, before update's pass starts)
bool update_follows_res(const op_arg *r, op_set set, const op_arg *u) {
  op_dat res = r[6].dat;
  return set == res->set && u[2].dat == res && u[0].dat != res && u[1].dat != res &&
         u[3].dat != res;
}

// save_soln(q -> qold') after update(qold, q, res, adt) on the same set: it
// copies the q update just wrote, at the same cell, to a dataset that is
// none of q, res, adt (update's qold is allowed: update reads it at the cell
// before the copy overwrites it)
bool save_follows_update(const op_arg *u, op_set uset, op_set set, const op_arg *sv) {
  return set == uset && sv[0].dat == u[1].dat && !dat_in(sv[1].dat, {u[1].dat, u[2].dat, u[3].dat});
}

// the update may wait for the next call only when its reduction need not
// reach the host before its own call returns
bool update_holdable() { return rt().gbl_deferred && rt().reduction == OP2B_REDUCE_TREE; }

bool res_holdable() {
  return effective_strategy("res_calc") == OP2B_STRATEGY_GATHER && tuning("gather_flux", 1);
}

// ---- loops run ahead of their calls --------------------------------------
// An update whose reduction must reach the caller before its call returns
// (reductions not deferred) cannot wait for the adt_calc the app calls next,
// nor, at the end of an outer iteration, for the next save_soln.  The update's
// per-cell pass computes them anyway, from the q it has just produced, into
// spare device buffers of adt (and of save_soln's output); the datasets
// themselves are left as they were.  When the expected call comes with the
// same arguments (and the constants unchanged), its result is already
// there: the dataset's device buffer and its spare swap, and no kernel runs.
// Any other call drops what was run ahead.  The observable state -- every
// dataset's device buffer between calls -- is the state without run-ahead.
// Whether save_soln follows is predicted from the updates before: airfoil's
// two updates per iteration alternate (adt_calc next, then save_soln next).
// Not while a captured graph exists (graphs hold dataset pointers).
struct Ahead {
  bool adt = false, save = false;
  std::vector<op_arg> adt_args, save_args;
  unsigned consts_version = 0;
};
Ahead g_ahead;
std::vector<op_arg> g_seen_adt, g_seen_save;  // the last adt_calc / save_soln calls
// The next res_calc + bres_calc's flux pass runs ahead too, queued behind
// the update's per-cell pass: it reads q as the update leaves it and adt from
// the spare buffer the update has just filled, so it is valid once that
// adt_calc is committed and the res_calc and bres_calc calls repeat the last
// ones.  The update's reduction is waited for on an event before it, so the
// flux pass runs while the host returns the rms and takes the next calls.
std::vector<op_arg> g_seen_res, g_seen_bres;  // the last res_calc / bres_calc calls
op_set g_seen_res_set = nullptr, g_seen_bres_set = nullptr;
std::vector<op_arg> g_seen_upd;  // the last airfoil update call (for the autotuner)
op_set g_seen_upd_set = nullptr;
struct NextFlux {
  bool valid = false, adt_committed = false;
  std::vector<op_arg> res_args, bres_args;
  op_set res_set = nullptr, bres_set = nullptr;
  unsigned consts_version = 0;
};
NextFlux g_next;
std::vector<op_arg> g_expect_bres;  // after a res_calc whose flux ran ahead
op_set g_expect_bres_set = nullptr;
cudaEvent_t g_fold_done = nullptr;
// jac1: the res that follows an update runs ahead the same way, into a
// spare buffer of du, and is swapped in when the res call repeats the last
// one with the same beta
std::vector<op_arg> g_seen_jres;
// the res call's beta (gbl OP_READ), copied when the call is recorded: the
// caller's variable may be gone by the next update, so g_seen_jres[3].data
// points here, never at the caller's memory
alignas(16) char g_seen_jres_beta[16];
op_set g_seen_jres_set = nullptr;
int g_seen_jres_variant = 0;
std::string g_seen_jres_name;
struct JacNext {
  bool valid = false;
  std::vector<op_arg> args;
  op_set set = nullptr;
  float beta = 0.f;
};
JacNext g_jnext;
unsigned g_save_after = 0;  // bit i: a save_soln came after the i-th latest update
std::vector<void *> g_spare;  // per dataset index

bool same_args(const std::vector<op_arg> &a, const op_arg *b) {
  for (size_t i = 0; i < a.size(); i++)
    if (a[i].argtype != b[i].argtype || a[i].dat != b[i].dat || a[i].map != b[i].map ||
        a[i].idx != b[i].idx || a[i].acc != b[i].acc || a[i].dim != b[i].dim)
      return false;
  return true;
}

void *spare_of(op_dat d) {
  if (g_spare.size() <= (size_t)d->index) g_spare.resize(d->index + 1, nullptr);
  if (!g_spare[d->index]) g_spare[d->index] = dev_alloc((size_t)d->size * d->set->size);
  return g_spare[d->index];
}

// the spare buffer becomes the dataset's, the dataset's old buffer the spare
void swap_in(op_dat d) {
  void *old = d->data_d;
  d->data_d = static_cast<char *>(g_spare[d->index]);
  g_spare[d->index] = old;
}

// res_calc, bres_calc, update whose rms is returned now: run the next
// adt_calc (and save_soln) ahead; false when that does not apply
bool run_chain_ahead(const std::vector<Held> &ch) {
  if (!tuning("run_ahead", 1) || rt().gbl_deferred || live_graphs() > 0 ||
      !tuning("gather_slots", 1))
    return false;
  const Held &u = ch[2];
  const op_arg *ua = u.args.data();
  if (g_seen_adt.size() != 6 || !adt_follows_update(ua, u.set, g_seen_adt[4].dat->set,
                                                    g_seen_adt.data()))
    return false;
  // save_soln predicted from the update two before this one (bit 0 is this
  // update, bit 1 the previous one)
  const bool save = ((g_save_after >> 2) & 1) && g_seen_save.size() == 2 &&
                    save_follows_update(ua, u.set, g_seen_save[0].dat->set, g_seen_save.data()) &&
                    !dat_in(g_seen_save[1].dat, {g_seen_adt[0].dat, g_seen_adt[1].dat,
                                                 g_seen_adt[2].dat, g_seen_adt[3].dat});
  void *adt_out = spare_of(g_seen_adt[5].dat);
  void *save_out = save ? spare_of(g_seen_save[1].dat) : nullptr;
  if (error_pending()) return false;
  std::vector<GblRequest> held;
  if (!run_res_chain(nullptr, ch[0].set, ch[0].args.data(), ch[1].set, ch[1].args.data(), ua,
                     g_seen_adt.data(), save ? g_seen_save.data() : nullptr, adt_out, save_out,
                     ch[0].flux_done, &held, ch[0].res_zero))
    return false;
  g_ahead.adt = true;
  g_ahead.save = save;
  g_ahead.adt_args = g_seen_adt;
  g_ahead.save_args = g_seen_save;
  g_ahead.consts_version = rt().consts_version;
  // the next chain's flux pass, behind an event that marks this update done
  const bool next = tuning("flux_ahead", 1) && g_seen_res.size() == 8 &&
                    g_seen_bres.size() == 6 && g_seen_res[2].dat == ua[1].dat &&
                    g_seen_res[3].dat == ua[1].dat && g_seen_res[4].dat == ua[3].dat &&
                    g_seen_res[5].dat == ua[3].dat && g_seen_res[6].dat == ua[2].dat &&
                    bres_follows_res(g_seen_res.data(), g_seen_bres.data()) &&
                    g_seen_adt[5].dat == ua[3].dat;
  if (!next) {
    red_finish(held);
    return true;
  }
  if (!g_fold_done) OP2B_CUDA(cudaEventCreateWithFlags(&g_fold_done, cudaEventDisableTiming));
  OP2B_CUDA(cudaEventRecord(g_fold_done, rt().stream));
  g_next = NextFlux();
  g_next.valid = run_res_flux_ahead(g_seen_res_set, g_seen_res.data(), g_seen_bres_set,
                                    g_seen_bres.data(), ua[3].dat, adt_out);
  g_next.res_args = g_seen_res;
  g_next.bres_args = g_seen_bres;
  g_next.res_set = g_seen_res_set;
  g_next.bres_set = g_seen_bres_set;
  g_next.consts_version = rt().consts_version;
  red_finish_after(g_fold_done, held);
  return true;
}

// jac update whose sum and max go back now: queue the next res behind it
bool jac_update_ahead(char const *name, op_set set, const op_arg *a, int variant) {
  if (!tuning("run_ahead", 1) || rt().gbl_deferred || live_graphs() > 0 || variant != 1 ||
      g_seen_jres.size() != 4 || g_seen_jres_variant != 1 ||
      g_seen_jres[1].dat != a[2].dat || g_seen_jres[2].dat != a[1].dat)
    return false;
  if (!can_run_jac_res_ahead(g_seen_jres_name.c_str(), g_seen_jres_set, g_seen_jres.data(), 1))
    return false;
  void *du_out = spare_of(a[1].dat);
  if (error_pending()) return false;
  std::vector<GblRequest> held;
  run_jac_update(name, set, a, variant, &held);
  if (error_pending()) {
    red_finish(held);
    return true;
  }
  if (!g_fold_done) OP2B_CUDA(cudaEventCreateWithFlags(&g_fold_done, cudaEventDisableTiming));
  OP2B_CUDA(cudaEventRecord(g_fold_done, rt().stream));
  g_jnext = JacNext();
  g_jnext.beta = *(const float *)g_seen_jres[3].data;  // the value the run uses
  g_jnext.valid = run_jac_res_ahead(g_seen_jres_name.c_str(), g_seen_jres_set,
                                    g_seen_jres.data(), 1, du_out);
  g_jnext.args = g_seen_jres;
  g_jnext.set = g_seen_jres_set;
  red_finish_after(g_fold_done, held);
  return true;
}

// run a chain, fused as far as the kernels allow
void run_chain(const std::vector<Held> &ch, const Held *adt) {
  if (ch.size() == 4) {  // res_calc, bres_calc, update, save_soln
    const Held &sv = ch[3];
    if (adt && tuning("gather_slots", 1) &&
        run_res_chain(nullptr, ch[0].set, ch[0].args.data(), ch[1].set, ch[1].args.data(),
                      ch[2].args.data(), adt->args.data(), sv.args.data(), nullptr, nullptr,
                      false, nullptr, ch[0].res_zero))
      return;
    run_chain(std::vector<Held>(ch.begin(), ch.begin() + 3), nullptr);
    run_chain(std::vector<Held>{sv}, adt);
    return;
  }
  if (ch.size() == 3 && !adt && ch[2].kind == K_AUPDATE) {
    g_save_after <<= 1;  // a new update: what follows it is not known yet
    if (run_chain_ahead(ch)) return;
  }
  const Held &h0 = ch[0];
  const op_arg *a0 = h0.args.data();
  if (ch.size() == 1) {
    if (adt && h0.kind == K_SAVE && run_save_adt(h0.set, a0, adt->args.data())) return;
    if (adt && h0.kind == K_AUPDATE && run_update_adt(h0.set, a0, adt->args.data())) return;
    run_kind(h0.kind, 0, h0.name.c_str(), h0.set, a0);
  } else {
    const Held &h1 = ch[1];
    const Held *u = ch.size() > 2 ? &ch[2] : nullptr;
    if (u && tuning("gather_slots", 1) &&
        run_res_chain(nullptr, h0.set, a0, h1.set, h1.args.data(), u->args.data(),
                      adt ? adt->args.data() : nullptr, nullptr, nullptr, nullptr,
                      h0.flux_done && h1.kind == K_BRES, nullptr,
                      h0.kind == K_RES && h0.res_zero))
      return;
    if (!run_res_bres(h0.set, a0, h1.set, h1.args.data())) {
      run_kind(h0.kind, 0, h0.name.c_str(), h0.set, a0);
      run_kind(h1.kind, 0, h1.name.c_str(), h1.set, h1.args.data());
    }
    if (u) {
      if (adt && run_update_adt(u->set, u->args.data(), adt->args.data())) return;
      run_kind(u->kind, 0, u->name.c_str(), u->set, u->args.data());
    }
  }
  if (adt) run_kind(adt->kind, 0, adt->name.c_str(), adt->set, adt->args.data());
}

Held make_held(Kind k, char const *name, op_set set, int nargs, const op_arg *args) {
  Held h;
  h.kind = k;
  h.name = name;
  h.set = set;
  h.args.assign(args, args + nargs);
  return h;
}

// Offer the next loop to the held chain.  Returns true when it was taken
// (held or run fused); false when the caller must flush and run it.
bool extend_chain(Kind k, char const *name, op_set set, int nargs, const op_arg *a) {
  if (g_chain.empty()) return false;
  const Held &h0 = g_chain[0];
  const op_arg *pa = h0.args.data();
  const size_t n = g_chain.size();
  if (n == 1 && h0.kind == K_JUPDATE && k == K_JRES && nargs == 4) {
    // jac1: the held update, then this res, as one launch
    std::vector<Held> ch;
    std::swap(ch, g_chain);
    if (jac_res_variant(nargs, a) == 1 &&
        run_jac_step(ch[0].name.c_str(), ch[0].set, ch[0].args.data(), name, set, a))
      return true;
    run_chain(ch, nullptr);  // the update alone; the caller runs the res
    return false;
  }
  if (n == 1 && h0.kind == K_SAVE && k == K_ADT && set == h0.set) {
    // save_soln(q -> qold), adt_calc(x, q' -> adt)
    op_dat q = pa[0].dat, qold = pa[1].dat;
    if (dat_in(a[5].dat, {q, qold}) || a[0].dat == qold || a[1].dat == qold ||
        a[2].dat == qold || a[3].dat == qold || a[4].dat == qold)
      return false;
    Held adt = make_held(k, name, set, nargs, a);
    std::vector<Held> ch;
    std::swap(ch, g_chain);
    run_chain(ch, &adt);
    return true;
  }
  if (n == 1 && h0.kind == K_AUPDATE && k == K_ADT && adt_follows_update(pa, h0.set, set, a)) {
    Held adt = make_held(k, name, set, nargs, a);
    std::vector<Held> ch;
    std::swap(ch, g_chain);
    run_chain(ch, &adt);
    return true;
  }
  if (n == 1 && h0.kind == K_RES && k == K_BRES && bres_follows_res(pa, a)) {
    g_chain.push_back(make_held(k, name, set, nargs, a));
    if (!tuning("fuse_update", 1) || !tuning("gather_slots", 1)) flush_pending();
    return true;
  }
  if (n == 2 && k == K_AUPDATE && update_follows_res(pa, set, a)) {
    g_chain.push_back(make_held(k, name, set, nargs, a));
    if (!update_holdable()) flush_pending();
    return true;
  }
  if (n == 3 && k == K_ADT && adt_follows_update(g_chain[2].args.data(), g_chain[2].set, set, a)) {
    Held adt = make_held(k, name, set, nargs, a);
    std::vector<Held> ch;
    std::swap(ch, g_chain);
    run_chain(ch, &adt);
    return true;
  }
  // the next outer iteration's save_soln, then its adt_calc, join the update
  if (n == 3 && k == K_SAVE && tuning("fuse_save", 1) &&
      save_follows_update(g_chain[2].args.data(), g_chain[2].set, set, a)) {
    g_chain.push_back(make_held(k, name, set, nargs, a));
    return true;
  }
  if (n == 4 && k == K_ADT && adt_follows_update(g_chain[2].args.data(), g_chain[2].set, set, a) &&
      !dat_in(g_chain[3].args[1].dat, {a[0].dat, a[1].dat, a[2].dat, a[3].dat})) {
    Held adt = make_held(k, name, set, nargs, a);
    std::vector<Held> ch;
    std::swap(ch, g_chain);
    run_chain(ch, &adt);
    return true;
  }
  return false;
}

// loops that may start a chain
bool holdable(Kind k, int variant = 0) {
  if (!tuning("fuse", 1)) return false;
  if (k == K_SAVE) return true;
  // jac1's update waits for the next res (one launch for both) when its
  // reductions need not reach the host before its call returns
  if (k == K_JUPDATE) return variant == 1 && rt().gbl_deferred && tuning("jac_step", 1);
  if (k == K_RES) return res_holdable();
  if (k == K_AUPDATE) return update_holdable();
  return false;
}

}  // namespace

namespace op2b {
void ahead_drop() {
  g_ahead = Ahead();
  g_next = NextFlux();
  g_jnext = JacNext();
  for (Held &h : g_chain) h.flux_done = false;
}

void ahead_reset() {
  ahead_drop();
  known_zero_forget();
  g_seen_adt.clear();
  g_seen_save.clear();
  g_seen_res.clear();
  g_seen_bres.clear();
  g_expect_bres.clear();
  g_seen_res_set = g_seen_bres_set = g_expect_bres_set = nullptr;
  g_seen_upd.clear();
  g_seen_upd_set = nullptr;
  g_seen_jres.clear();
  g_seen_jres_set = nullptr;
  g_seen_jres_variant = 0;
  g_save_after = 0;
  for (void *p : g_spare) dev_free(p);
  g_spare.clear();
}

// the last res_calc, bres_calc, update and adt_calc calls, when they form
// the airfoil chain (bres_calc after res_calc, update after both, adt_calc
// after update): what the autotuner times
bool last_res_chain(ChainArgs *c) {
  if (g_seen_res.size() != 8 || g_seen_bres.size() != 6 || g_seen_upd.size() != 5 ||
      g_seen_adt.size() != 6 || !g_seen_res_set || !g_seen_bres_set || !g_seen_upd_set)
    return false;
  if (!bres_follows_res(g_seen_res.data(), g_seen_bres.data()) ||
      !update_follows_res(g_seen_res.data(), g_seen_upd_set, g_seen_upd.data()) ||
      !adt_follows_update(g_seen_upd.data(), g_seen_upd_set, g_seen_adt[4].dat->set,
                          g_seen_adt.data()))
    return false;
  c->rset = g_seen_res_set;
  c->bset = g_seen_bres_set;
  c->uset = g_seen_upd_set;
  c->aset = g_seen_adt[4].dat->set;
  c->ra = g_seen_res;
  c->ba = g_seen_bres;
  c->ua = g_seen_upd;
  c->aa = g_seen_adt;
  return true;
}

void flush_pending() {
  if (g_chain.empty()) return;
  std::vector<Held> ch;
  std::swap(ch, g_chain);
  run_chain(ch, nullptr);
}

// ------------------------------------------------- datasets known zero ----
// A dataset whose device buffer holds +0.0 in every element.  airfoil's
// update leaves res so (airfoil/update.h:9-11) and res_calc and bres_calc
// only add to it, so the next res chain's fold starts its sums from +0.0 in
// registers instead of reading res, and leaves res as it is instead of
// writing the zeros again: the same values, 32 bytes per cell less traffic.
// A flag is set when a chain whose update zeroes the dataset is enqueued and
// cleared by every loop call that names the dataset as written (before the
// loop is held or run), so it describes the device state once all work
// handed to the stream has run.  Datasets change only through the library's
// calls, as run-ahead assumes too.  A capture runs nothing: the flags are put
// back at its end and each launch of the graph applies its effect on them.
namespace {
std::vector<unsigned char> g_zero, g_zero_saved, g_zero_touched, g_zero_set_in_capture;
bool g_zero_capturing = false;
}  // namespace

bool dat_known_zero(op_dat d) {
  return d && d->index >= 0 && (size_t)d->index < g_zero.size() && g_zero[d->index];
}

void dat_set_known_zero(op_dat d, bool zero) {
  if (!d || d->index < 0) return;
  const size_t i = (size_t)d->index;
  if (g_zero.size() <= i) {
    if (!zero) return;
    g_zero.resize(i + 1, 0);
  }
  g_zero[i] = zero;
  if (g_zero_capturing) {
    if (g_zero_touched.size() <= i) g_zero_touched.resize(i + 1, 0);
    if (g_zero_set_in_capture.size() <= i) g_zero_set_in_capture.resize(i + 1, 0);
    g_zero_touched[i] = 1;
    if (zero) g_zero_set_in_capture[i] = 1;
  }
}

void known_zero_forget() {
  if (g_zero_capturing)
    for (size_t i = 0; i < g_zero.size(); i++)
      if (g_zero[i]) {
        if (g_zero_touched.size() <= i) g_zero_touched.resize(i + 1, 0);
        g_zero_touched[i] = 1;
      }
  std::fill(g_zero.begin(), g_zero.end(), 0);
}

void known_zero_capture_begin() {
  g_zero_saved = g_zero;
  g_zero_touched.clear();
  g_zero_set_in_capture.clear();
  g_zero_capturing = true;
}

std::vector<std::pair<int, unsigned char>> known_zero_capture_end() {
  std::vector<std::pair<int, unsigned char>> eff;
  if (!g_zero_capturing) return eff;
  for (size_t i = 0; i < g_zero_touched.size(); i++)
    if (g_zero_touched[i]) eff.emplace_back((int)i, i < g_zero.size() ? g_zero[i] : 0);
  g_zero = g_zero_saved;
  g_zero_capturing = false;
  return eff;
}

void known_zero_apply(const std::vector<std::pair<int, unsigned char>> &eff) {
  for (auto &e : eff) {
    if (g_zero.size() <= (size_t)e.first) g_zero.resize(e.first + 1, 0);
    g_zero[e.first] = e.second;
  }
}

bool known_zero_from_before_capture(op_dat d) {
  if (!g_zero_capturing || !d || d->index < 0) return false;
  const size_t i = (size_t)d->index;
  return i >= g_zero_set_in_capture.size() || !g_zero_set_in_capture[i];
}
}  // namespace op2b

namespace {
void par_loop_run(char const *name, op_set set, int nargs, const op_arg *args);
}

extern "C" void op2b_par_loop(char const *name, op_set set, int nargs, const op_arg *args) {
  // a restarted run before its checkpoint: hand back the saved values
  if (checkpoint_fast_forward() && checkpoint_before_loop(name, nargs, args)) {
    for (int m = 0; m < nargs; m++)  // the saved values replace what the loop writes
      if (args[m].argtype == OP_ARG_DAT && args[m].acc != OP_READ)
        dat_set_known_zero(args[m].dat, false);
    return;
  }
  par_loop_run(name, set, nargs, args);
  if (!error_pending()) checkpoint_after_loop(nargs, args);
}

namespace {
// the datasets a call writes may hold other values than zeros afterwards
void note_writes(int nargs, const op_arg *args) {
  for (int m = 0; m < nargs; m++)
    if (args[m].argtype == OP_ARG_DAT && args[m].acc != OP_READ)
      dat_set_known_zero(args[m].dat, false);
}

void par_loop_run(char const *name, op_set set, int nargs, const op_arg *args) {
  if (set == nullptr) {
    fail(1, "error: invalid set in kernel \"%s\"\n", name ? name : "(null)");
    return;
  }
  if (!rt().cuda_ready) {
    ensure_cuda();
    if (error_pending()) return;
  }
  if (renumber_enabled()) {
    renumber_apply();  // once, at the first loop: order the sets, move the data
    if (error_pending()) return;
  }
  // the checks op_seq.h runs when OP_diags > 0 (common/op_seq.h:37-39); a
  // device loop always runs them, since bad arguments would fault the GPU
  int ninds = 0;
  for (int m = 0; m < nargs; m++) {
    op_arg_check(set, m, args[m], &ninds, name);
    if (error_pending()) return;
    if (args[m].argtype == OP_ARG_DAT && (!args[m].dat || !args[m].dat->data_d)) {
      fail(1, "error: arg %d in kernel \"%s\"\ndataset has no device copy \n", m, name);
      return;
    }
  }
  if (OP_diags > 2) {
    if (ninds == 0) printf(" kernel routine w/o indirection:  %s \n", name);
    else printf(" kernel routine with indirection: %s \n", name);
  }
  int v;
  Kind k = classify(nargs, args, &v);
  if (k == K_NONE) {
    flush_pending();
    fail(1,
         "op2b error: no device implementation of loop \"%s\" with this argument signature "
         "(%d args)\n",
         name, nargs);
    return;
  }
  // res_calc: whether res holds zeros before this call adds to it
  bool res_zero = k == K_RES && dat_known_zero(args[6].dat);
  note_writes(nargs, args);
  if (k == K_ADT) g_seen_adt.assign(args, args + nargs);
  if (k == K_SAVE) {
    g_seen_save.assign(args, args + nargs);
    g_save_after |= 1;
  }
  if (k == K_RES) {
    g_seen_res.assign(args, args + nargs);
    g_seen_res_set = set;
  }
  if (k == K_AUPDATE) {
    g_seen_upd.assign(args, args + nargs);
    g_seen_upd_set = set;
  }
  if (k == K_BRES) {
    g_seen_bres.assign(args, args + nargs);
    g_seen_bres_set = set;
  }
  if (k == K_JRES) {
    if (g_jnext.valid && set == g_jnext.set && same_args(g_jnext.args, args) &&
        *(const float *)args[3].data == g_jnext.beta) {
      swap_in(args[2].dat);  // the res run ahead: its du is ready
      g_jnext = JacNext();
      return;
    }
    g_seen_jres.assign(args, args + nargs);
    const size_t beta_bytes =
        (size_t)args[3].dim * (args[3].type && strcmp(args[3].type, "double") == 0 ? 8 : 4);
    if (nargs == 4 && args[3].data && beta_bytes <= sizeof(g_seen_jres_beta)) {
      memcpy(g_seen_jres_beta, args[3].data, beta_bytes);
      g_seen_jres[3].data = g_seen_jres_beta;
    } else {
      g_seen_jres.clear();  // nothing recorded: no run-ahead for this res
    }
    g_seen_jres_set = set;
    g_seen_jres_variant = v;
    g_seen_jres_name = name;
  }
  g_jnext = JacNext();
  if (g_ahead.adt || g_ahead.save) {  // the call run ahead: swap its result in
    if (k == K_SAVE && g_ahead.save && same_args(g_ahead.save_args, args)) {
      swap_in(args[1].dat);
      g_ahead.save = false;
      return;
    }
    if (k == K_ADT && g_ahead.adt && same_args(g_ahead.adt_args, args) &&
        rt().consts_version == g_ahead.consts_version) {
      swap_in(args[5].dat);
      g_ahead = Ahead();
      g_next.adt_committed = true;
      return;
    }
    g_ahead = Ahead();
    g_next = NextFlux();
  }
  // the flux pass run ahead counts for this res_calc only if everything
  // since matched; a bres_calc other than the expected one undoes it
  bool res_flux_done = false;
  if (k == K_RES) {
    res_flux_done = g_next.valid && g_next.adt_committed && g_chain.empty() &&
                    set == g_next.res_set && same_args(g_next.res_args, args) &&
                    rt().consts_version == g_next.consts_version;
    g_expect_bres = g_next.bres_args;
    g_expect_bres_set = g_next.bres_set;
  }
  g_next = NextFlux();
  if (k == K_BRES && !g_chain.empty() && g_chain[0].kind == K_RES && g_chain[0].flux_done &&
      !(g_chain.size() == 1 && set == g_expect_bres_set && g_expect_bres.size() == 6 &&
        same_args(g_expect_bres, args)))
    g_chain[0].flux_done = false;
  if (!g_chain.empty()) {
    if (extend_chain(k, name, set, nargs, args)) return;
    flush_pending();
    // the chain just run may have zeroed res; this call's writes follow it
    if (k == K_RES) res_zero = dat_known_zero(args[6].dat);
    note_writes(nargs, args);
  }
  if (holdable(k, v)) {
    g_chain.push_back(make_held(k, name, set, nargs, args));
    if (k == K_RES) {
      g_chain.back().flux_done = res_flux_done;
      g_chain.back().res_zero = res_zero;
    }
    return;
  }
  if (k == K_JUPDATE && jac_update_ahead(name, set, args, v)) return;
  run_kind(k, v, name, set, args);
}
}  // namespace

extern "C" {

// the per-loop entry points of the generated app mains
// (airfoil/airfoil_op.cpp:64-99, jac1/jac_op.cpp:58-73)
void op_par_loop_save_soln(char const *name, op_set set, op_arg a0, op_arg a1) {
  op_arg args[2] = {a0, a1};
  op2b_par_loop(name, set, 2, args);
}
void op_par_loop_adt_calc(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                          op_arg a3, op_arg a4, op_arg a5) {
  op_arg args[6] = {a0, a1, a2, a3, a4, a5};
  op2b_par_loop(name, set, 6, args);
}
void op_par_loop_res_calc(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                          op_arg a3, op_arg a4, op_arg a5, op_arg a6, op_arg a7) {
  op_arg args[8] = {a0, a1, a2, a3, a4, a5, a6, a7};
  op2b_par_loop(name, set, 8, args);
}
void op_par_loop_bres_calc(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                           op_arg a3, op_arg a4, op_arg a5) {
  op_arg args[6] = {a0, a1, a2, a3, a4, a5};
  op2b_par_loop(name, set, 6, args);
}
void op_par_loop_update(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                        op_arg a3, op_arg a4) {
  op_arg args[5] = {a0, a1, a2, a3, a4};
  op2b_par_loop(name, set, 5, args);
}
void op_par_loop_res(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2, op_arg a3) {
  op_arg args[4] = {a0, a1, a2, a3};
  op2b_par_loop(name, set, 4, args);
}

}  // extern "C"
