// plan.h -- device execution plans (not installed).
#pragma once

#include <memory>
#include <vector>

#include "internal.h"

namespace op2b {

// The reference's execution plan (common/op_lib_core.h:122-150), built on the
// device by build_plan() and kept there.  Arrays follow the reference's
// definitions exactly; `pub` is the op_plan view handed to callers of
// op_plan_get (device pointers except ncolblk and nindirect).
struct DevPlan {
  // cache key (common/op_lib_core.c:632-659)
  std::string name;
  op_set set = nullptr;
  int part_size = 0, nargs = 0, ninds = 0;
  std::vector<op_dat> dats;
  std::vector<op_map> maps;
  std::vector<int> idxs, inds;
  std::vector<op_access> accs;

  int bsize = 0, nblocks = 0, ncolors = 0, nshared = 0;
  int *d_nthrcol = nullptr, *d_thrcol = nullptr, *d_offset = nullptr, *d_nelems = nullptr;
  int *d_ind_offs = nullptr, *d_ind_sizes = nullptr, *d_blkmap = nullptr;
  std::vector<int *> d_ind_maps;
  std::vector<short *> d_loc_maps;
  std::vector<int> nindirect, ncolblk, colstart;  // host
  std::vector<int> nthrcol_h;                     // host copy (for diagnostics)
  double transfer = 0, transfer2 = 0, transfer3 = 0;
  float avg_thread_colours = 0;
  int max_thread_colours = 0;
  op_plan pub;
  std::vector<int *> pub_ind_maps;
  std::vector<short *> pub_loc_maps;
  int count = 0;
};

// Owner-computes ("gather") plan for one group of OP_INC arguments that
// increment the same dataset: for every target element, the list of
// (element, slot) contributions in ascending order, slot = position of the
// argument inside the group.  This is the order of the sequential back-end
// (common/op_seq.h:26-57, element loop outermost, arguments in kernel order).
struct GatherPlan {
  op_set set = nullptr;           // loop set
  op_dat dat = nullptr;           // incremented dataset
  std::vector<op_map> maps;       // per slot
  std::vector<int> idxs;          // per slot
  int nslots = 0;
  int ntarget = 0;                // size of dat->set
  int nactive = 0;                // targets with at least one contribution
  int *d_row = nullptr;           // [nactive + 1] offsets into d_keys
  int *d_keys = nullptr;          // [set->size * nslots] element * nslots + slot
  int *d_active = nullptr;        // [nactive] target ids, nullptr when all active
  int max_row = 0;
  // CTA tiles for the contribution-parallel kernels: tile b owns the
  // targets whose first contribution lies in [kTile*b, kTile*(b+1)), i.e.
  // targets [d_tile_first[b], d_tile_first[b+1]); [ntiles + 1] entries
  int ntiles = 0;
  int *d_tile_first = nullptr;
  long long nkeys = 0;
  // per-element contribution buffer of the two-pass kernels, allocated on
  // first use (outside any graph capture) and kept with the plan
  void *d_contrib = nullptr;
  size_t contrib_bytes = 0;
};

// contributions per CTA tile of the contribution-parallel gather kernels
constexpr int kTile = 256;

// Fixed-width (ELL) contribution lists for an edge loop `a` with two
// increment arguments (slot 0 adds the edge's value, slot 1 subtracts it),
// optionally followed by a loop `b` with one (adds): the kernels store one
// value per edge of a in v[0, na), one per element of b in v[na, na+nb),
// and -0.0 in v[na+nb].  Target t owns entries ell[t*width, (t+1)*width):
// (index << 1 | negate) of its contributions, a's in a's ascending order
// then b's in b's order, padded with (na+nb) << 1.  Adding the entries in
// list order is the order of the sequential back-end running a then b;
// -0.0 is the exact identity of IEEE addition and r + (-v) equals r - v.
struct ChainSched;  // airfoil.cu: the persistent chain's work queue over these lists
struct TilePlan;    // airfoil.cu: the tiled chain's per-tile flux lists
struct SlotPlan {
  const GatherPlan *a = nullptr, *b = nullptr;
  int ntarget = 0;
  int width = 0;            // max contributions of one target
  int na = 0, nb = 0;       // elements of a and b
  int *d_ell = nullptr;     // [ntarget * width]
  void *d_buf = nullptr;    // the (na + nb + 1) values, allocated by the loop
  size_t buf_bytes = 0;
  ChainSched *chain = nullptr;  // built by the first persistent chain launch
  bool chain_unsuited = false;  // a cell tile reads too many flux tiles for it
  TilePlan *tile = nullptr;     // built by the first tiled chain launch
  bool tile_unsuited = false;   // no tile size fits shared memory
};
// free a slot plan's persistent-chain queue and tile plan (airfoil.cu)
void release_chain_sched(SlotPlan *sp);
void release_tile_plan(SlotPlan *sp);

// widest list the fold kernels accept
constexpr int kMaxSlotWidth = 8;

// Find or build the lists of a (two slots) and b (nullable, one slot);
// nullptr when some target has more than kMaxSlotWidth contributions or the
// padding would more than double the lists (the caller then uses the CSR
// fold).
SlotPlan *get_slot_plan(const GatherPlan *a, const GatherPlan *b);

// Find or build the reference-compatible plan (device resident).
DevPlan *get_plan(char const *name, op_set set, int part_size, int nargs, const op_arg *args,
                  int ninds, const int *inds);
// Find or build the gather plan for the INC args listed in slots (all on
// the same dat).
GatherPlan *get_gather_plan(op_set set, const op_arg *args, const std::vector<int> &slots);
// Device validation of a plan; returns the number of violations.
long validate_plan(const DevPlan &p);

// device-wide exclusive scan of n ints (in place allowed); returns the total
long long exclusive_scan(const int *d_in, int *d_out, int n, cudaStream_t s);
// the same, queued only (no total, no host wait)
void exclusive_scan_nosync(const int *d_in, int *d_out, int n, cudaStream_t s);

}  // namespace op2b
