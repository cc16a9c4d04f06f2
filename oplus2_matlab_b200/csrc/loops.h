// loops.h -- host-side pieces shared by the loop implementations.
#pragma once

#include <vector>

#include "internal.h"
#include "plan.h"

namespace op2b {

// device view of one argument's indirection: element e -> map[idx + e*dim],
// or e itself when map == nullptr (OP_ID)
struct IdxMap {
  const int *map;
  int dim, idx;
};

inline IdxMap idx_map(const op_arg &a) {
  IdxMap m{nullptr, 0, 0};
  if (a.map) {
    m.map = map_dev(a.map);
    m.dim = a.map->dim;
    m.idx = a.idx;
  }
  return m;
}

// strategy actually used for a loop with OP_INC through a map
int effective_strategy(char const *loop_name);

// algorithmic (compulsory) bytes of one loop call: every distinct map array
// once, every distinct dataset once, read-write and increment data twice
double compulsory_bytes(op_set set, int nargs, const op_arg *args);

// -------------------------------------------------- global reductions -----
enum GblType { GBL_F32 = 0, GBL_F64 = 1 };
struct GblRequest {
  char *host;      // caller's variable (op_arg.data)
  int slot;        // result slot in the device ring
  op_access acc;
  int type;        // GblType
  bool assign;     // SEQ-mode sum: device value already includes the seed
};
constexpr int kMaxRedBlocks = 4096;
void *red_partials(int i);       // [kMaxRedBlocks] of 8-byte entries, i in {0,1}
unsigned *red_ticket();
void *red_slot_ptr(int slot);    // 8-byte device slot
int red_new_slot();
void *red_seq_buffer(size_t bytes);  // scratch for SEQ-mode contributions
void red_finish(const std::vector<GblRequest> &reqs);
// the same, waiting only for the work up to the event (not deferred mode)
void red_finish_after(cudaEvent_t done, const std::vector<GblRequest> &reqs);
// deferred requests (graph capture): count, take those added since a mark,
// and re-arm a set (replacing any pending request on the same slots)
size_t red_pending_count();
std::vector<GblRequest> red_take_pending_since(size_t mark);
void red_replace_pending(const std::vector<GblRequest> &reqs);
// keep every slot handed out so far out of reuse (they are baked into a graph)
void red_reserve_for_graph();
int red_grid(long long n, int threads);  // fixed grid for a set size

// loop implementations (airfoil.cu, jac.cu)
void run_save_soln(char const *name, op_set set, const op_arg *args);
void run_adt_calc(char const *name, op_set set, const op_arg *args);
void run_res_calc(char const *name, op_set set, const op_arg *args);
void run_bres_calc(char const *name, op_set set, const op_arg *args);
void run_airfoil_update(char const *name, op_set set, const op_arg *args);
void run_jac_res(char const *name, op_set set, const op_arg *args, int variant);
// held: the reductions are appended there for the caller to deliver
void run_jac_update(char const *name, op_set set, const op_arg *args, int variant,
                    std::vector<GblRequest> *held = nullptr);
// jac1's res into du_out (a spare buffer of du's size) instead of du, ahead
// of its call; false when not applicable (nothing launched)
// jac1's update followed by its res as one launch (jac.cu); false when the
// shapes do not suit it
bool run_jac_step(char const *uname, op_set uset, const op_arg *ua, char const *rname,
                  op_set rset, const op_arg *ra);
bool run_jac_res_ahead(char const *name, op_set set, const op_arg *args, int variant,
                       void *du_out);
// whether run_jac_res_ahead would launch for these arguments (GATHER, jac1,
// every node a target); allocates nothing beyond the res loop's own plan
bool can_run_jac_res_ahead(char const *name, op_set set, const op_arg *args, int variant);

// the last airfoil res_calc chain's calls (loops.cpp), for the autotuner
struct ChainArgs {
  op_set rset = nullptr, bset = nullptr, uset = nullptr, aset = nullptr;
  std::vector<op_arg> ra, ba, ua, aa;
};
bool last_res_chain(ChainArgs *c);

// fused loop pairs (airfoil.cu); false = not applicable, run them separately
bool run_save_adt(op_set set, const op_arg *save_args, const op_arg *adt_args);
bool run_update_adt(op_set set, const op_arg *update_args, const op_arg *adt_args);
bool run_res_bres(op_set res_set, const op_arg *res_args, op_set bres_set,
                  const op_arg *bres_args);
// res_calc, then optionally bres_calc, update and adt_calc (each nullable,
// in that nesting), through per-cell increment slots; false when the mesh
// does not suit slots (nothing has run).  save_args: save_soln between
// update and adt_calc (the next outer iteration's first loops), storing the
// new q to its output as well; needs update and adt_calc, else false.
// adt_out / save_out (device buffers of adt's and save_soln's output size,
// or nullptr): adt_calc's and save_soln's values go there instead of into
// their datasets.  name: the timer name, or nullptr for the joined loop names.
// flux_done: the flux pass already ran for exactly these arguments (run
// ahead, run_res_flux_ahead).  held: the update's reduction is appended
// there for the caller to deliver, instead of being delivered here.
// res_zero: res held +0.0 in every element when res_calc was called (then,
// with update, res is neither read nor rewritten).
bool run_res_chain(char const *name, op_set res_set, const op_arg *res_args, op_set bres_set,
                   const op_arg *bres_args, const op_arg *update_args, const op_arg *adt_args,
                   const op_arg *save_args = nullptr, void *adt_out = nullptr,
                   void *save_out = nullptr, bool flux_done = false,
                   std::vector<GblRequest> *held = nullptr, bool res_zero = false);
// the flux pass of a res_calc + bres_calc chain before its calls, adt read
// from adt_now instead of adt's buffer; false when not applicable
bool run_res_flux_ahead(op_set res_set, const op_arg *res_args, op_set bres_set,
                        const op_arg *bres_args, op_dat adt, const void *adt_now);
void release_fused_plans();

}  // namespace op2b
