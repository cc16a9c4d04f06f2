// internal.h -- shared declarations of libop2b200 (not installed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "op2b.h"
#include "op_lib.h"

extern "C" int OP_cache_line_size;  // common/op_lib_core.c:43, not in op_lib.h

namespace op2b {

// ---------------------------------------------------------------- errors --
// Print like the reference (printf + exit) in EXIT mode; in RETURN mode print,
// remember the message and let the caller return a neutral value.
void fail(int exit_code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
bool error_pending();  // a fail() happened since the last clear (RETURN mode)

void cuda_fail(cudaError_t err, const char *what, const char *file, int line);
#define OP2B_CUDA(call)                                                    \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) ::op2b::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

// ------------------------------------------------------------ device data --
struct MapDev {
  int *d = nullptr;  // device copy of map->map, same layout (from-major, dim-minor)
};

struct DatDev {
  size_t bytes = 0;  // set->size * dat->size
};

// per-loop timing record (op_kernel of the reference plus device events)
// per-loop timing record (op_kernel of the reference plus device events).
// Sampled timing (the default) times a loop's first call and every
// kTimingSample-th call after it; the total is the first call's time plus
// the sampled mean times the other calls.
constexpr int kTimingSample = 16;
struct LoopTimer {
  std::string name;
  int kernel_index = -1;  // slot in OP_kernels
  struct Timed {
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    bool first;
  };
  std::vector<Timed> pending;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> free_pairs;
  double seconds = 0.0;   // estimated total device time
  double first_s = 0.0, sampled_s = 0.0;
  long long sampled_n = 0;
  int count = 0;
};

struct Runtime {
  bool cuda_ready = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int strategy = OP2B_STRATEGY_AUTO;
  int reduction = OP2B_REDUCE_TREE;
  int error_mode = OP2B_ERRORS_EXIT;
  bool gbl_deferred = false;
  int timing = 1;  // 0 off, 1 sampled (every kTimingSample-th call), 2 every call
  int num_sms = 148;
  int smem_optin = 48 * 1024;  // dynamic shared memory a CTA may opt in to
  std::string device_name;  // queried once per process (the query takes milliseconds)

  std::vector<MapDev> maps;  // by op_map index
  std::vector<DatDev> dats;  // by op_dat index

  // constants declared by op_decl_const_char, by name (raw bytes + type)
  struct Const {
    std::string type;
    int dim = 0, size = 0;
    std::vector<char> bytes;
  };
  std::map<std::string, Const> consts;
  unsigned consts_version = 0;

  std::map<std::string, LoopTimer> timers;

  // kernel variant knobs (op2b_set_tuning), read by the loop launchers
  std::map<std::string, int> tuning;

  // stream capture in progress (graph.cu): per-loop event pairs recorded
  // into the graph when profiling
  bool capture_profile = false;
  struct CapturedLoop {
    std::string name;
    cudaEvent_t start, stop;
  };
  std::vector<CapturedLoop> capture_events;

  // device scratch for global reductions: partials + final slots
  void *red_scratch = nullptr;
  size_t red_scratch_bytes = 0;
  void *red_host = nullptr;  // pinned mirror of the final slots
  size_t red_host_bytes = 0;

  // deferred global reductions waiting for the next sync
  struct DeferredGbl {
    char *host;        // user variable
    int bytes_offset;  // offset of the result in red_host
    int dim;
    op_access acc;
    int is_double;
  };
  std::vector<DeferredGbl> deferred;
};

Runtime &rt();

// value of a tuning knob, or `def` when unset
inline int tuning(const char *key, int def) {
  auto it = rt().tuning.find(key);
  return it == rt().tuning.end() ? def : it->second;
}

// device copy of a map, uploaded on first use
const int *map_dev(op_map m);

// launch the loop held back for fusion, if any (loops.cpp); every call that
// needs device results to be complete or issued runs it first
void flush_pending();

// device memory helpers (long-lived allocations)
void *dev_alloc(size_t bytes);
void dev_free(void *p);
// stream-ordered scratch from the library's pool; free with cudaFreeAsync
cudaError_t pool_malloc_async(void **p, size_t bytes, cudaStream_t s);
// a map's device copy queued at its declaration (nullptr: none, the first
// loop that uses the map makes it), handed to the map once it is valid,
// or dropped when the declaration fails
void *map_upload_begin(const int *imap, size_t bytes);
void map_upload_attach(op_map m, void *d);
void map_upload_abort(void *d);
void ensure_cuda();  // op_init's device part, also run lazily

// timing around one loop call
struct LoopScope {
  LoopTimer *t = nullptr;
  std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
  bool captured = false, first = false;
  LoopScope(char const *name, double transfer, double transfer2);
  ~LoopScope();
};
void flush_timers();  // harvest finished event pairs into OP_kernels

// event pair around one kernel of a fused loop chain, recorded only inside a
// profiled graph capture (it adds no entry to the op_timing_output table)
struct PhaseScope {
  explicit PhaseScope(const std::string &name);
  ~PhaseScope();

 private:
  std::string name_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
};

// constants lookup: copies up to n values of the named constant into out,
// converted to T; returns the number found (0 if never declared)
int const_get_f32(char const *name, float *out, int n);
int const_get_f64(char const *name, double *out, int n);

// loops run ahead of their calls (loops.cpp): after an update whose result
// must reach the caller, the next adt_calc (and save_soln) run in the
// update's kernel into spare buffers, swapped in when the calls come
void ahead_drop();   // discard what was run ahead (constants, capture, restore)
void ahead_reset();  // op_exit: also free the spare buffers
void noalloc_reset();  // op_exit: forget op2b_update_noalloc's cached scratch addresses
int live_graphs();   // captured graphs not yet destroyed (graph.cu)
// A dataset's second device buffer (allocated on first use) and the swap
// of the two, for loops that write a dataset other elements of the same
// launch still read (airfoil.cu); swaps made while capturing are counted
void *alt_of(op_dat d);
void flip(op_dat d, bool capturing);
// Datasets known to hold +0.0 in every element of their device buffer
// (loops.cpp): set when a res chain whose update zeroes res is enqueued,
// cleared by every loop call that writes the dataset
bool dat_known_zero(op_dat d);
void dat_set_known_zero(op_dat d, bool zero);
void known_zero_forget();  // any dataset may have changed (restore, renumbering, op_exit)
// a capture runs nothing: the flags are saved at its start and put back at
// its end, which returns the capture's effect on them (dataset index, flag)
// for each launch of the graph to apply
void known_zero_capture_begin();
std::vector<std::pair<int, unsigned char>> known_zero_capture_end();
void known_zero_apply(const std::vector<std::pair<int, unsigned char>> &effects);
// capturing, and no captured work has set d's flag: a kernel that relies on
// d's zeros (seen when its loop was called) relies on the state before the
// capture
bool known_zero_from_before_capture(op_dat d);
// graph.cu: the kernel just captured skips reading d (its kernel parameter
// `arg` of `nparams`) because d was zero when the capture began; a launch of
// the graph when d may hold other values hands the kernel d's buffer instead
// and, when read_kernel is not null, runs read_kernel (the same parameters)
// on read_grid CTAs in its place
void capture_zero_entry(op_dat d, int arg, int nparams, void *buf, const void *read_kernel,
                        int read_grid);
void tile_capture_begin();  // graph capture: count the tiled chain's buffer swaps
void tile_capture_end();    // ... and undo an odd count inside the graph
void release_tile_alts();   // op_exit: free the tiled chain's second buffers
// The tiled res_calc chain's lists (airfoil.cu): for tiles of ct consecutive
// cells, each tile's distinct list indices ascending (tflux, tile t's run at
// toff[t]) and each list entry as (slot in its tile's run << 1 | side)
struct TileLists {
  int ct = 0, ntile = 0, maxcnt = 0;  // cells per tile, tiles, the longest run (-1: on the device)
  int *toff = nullptr, *tflux = nullptr, *tell = nullptr;
  int *d_longest = nullptr;  // the longest run, when built asynchronously
};
bool build_tile_lists(const int *ell, int ncell, int W, int ct, cudaStream_t s, TileLists *out);
bool build_tile_lists_async(const int *ell, int ncell, int W, int ct, cudaStream_t s,
                            TileLists *out);
int tile_lists_longest(TileLists *tl, cudaStream_t s);
void free_tile_lists(TileLists *tl, cudaStream_t s);
// sorts the m 64-bit keys at a (m a power of two) ascending on stream s
bool sort_keys_u64(unsigned long long *a, long long m, cudaStream_t s);

// renumbering of the sets for locality (renumber.cu)
bool renumber_enabled();
void renumber_apply();                 // first loop call: order the sets, move the data
void renumber_reset();                 // op_exit
const int *perm_new2old_dev(op_set s);  // device permutation, nullptr when not renumbered
const int *perm_old2new_dev(op_set s);
void permute_dat_in_place(op_dat d);   // a dataset declared after renumbering
bool fetch_unpermuted(op_dat d, void *host);  // false: not renumbered, nothing done
bool renumber_map_device(op_map m, int *d_map);  // false: map unchanged

// op_checkpoint (checkpoint.cpp): fast-forward of a restarted run, and the
// log of reduction values returned to the app
bool checkpoint_fast_forward();
bool checkpoint_before_loop(char const *name, int nargs, const op_arg *args);  // true: skip
void checkpoint_after_loop(int nargs, const op_arg *args);
void checkpoint_reset();  // op_exit

// global reductions: device slot management (reduce.cu)
void deliver_deferred();

}  // namespace op2b
