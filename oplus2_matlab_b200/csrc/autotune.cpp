// autotune.cpp -- the plain path's autotuner (op2b_autotune).
//
// The reference leaves the launch shape of each loop to compile-time macros
// (OP_PART_SIZE_n and OP_BLOCK_SIZE_n in the generated stubs,
// airfoil/res_calc_kernel.cu:181-204) and to op_plan_core's 48 KB rule
// (common/op_lib_core.c:663-673); its developer notes expect autotuning of
// those choices to be worth a factor of two (doc/dev.tex:975-990).  Here the
// choices are the library's tuning knobs for the dominant chain,
// res_calc + bres_calc + update + adt_calc, and they are chosen by timing
// them on the app's own mesh and data.
//
// op2b_autotune(cache, iters), called after one outer iteration of the app
// has run through the loop API (so the chain's calls are known):
//  1. looks the chain up in the cache file (device, real type, set sizes);
//     a hit applies the stored knobs and returns 1 without timing;
//  2. otherwise saves q, res and adt, and for every candidate setting runs
//     the chain once untimed (plans and queues are built then), then times
//     `iters` launches, each after an L2 flush, with CUDA events; the data
//     is put back after every candidate, so the app's state is untouched;
//  3. applies the fastest setting, appends it to the cache, returns 0.
//
// Every candidate leaves q, qold, res and adt bit-identical (they change
// the launch shape, not the per-element arithmetic or the order in which a
// cell's contributions are added): the persistent one-launch chain against
// the flux pass + per-cell pass, its flux tile size, cells per thread and
// queue lag, the per-cell pass variants.  They do change the order of the
// TREE rms sum (its tree follows the launch shape), as any launch shape
// does.  With allow_reorder != 0 the reference's colouring scheme
// (COLOURED) is timed too, at part sizes 64..512: it adds a cell's
// contributions in colour order, so its fields differ from op_seq.h's in
// the last bits; it is chosen only if it is faster.

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <utility>
#include <vector>

#include "internal.h"
#include "loops.h"

namespace op2b {
namespace {

typedef std::vector<std::pair<std::string, int>> Knobs;

struct Candidate {
  Knobs knobs;
  int strategy = OP2B_STRATEGY_GATHER;
  int part_size = 0, block_size = 0;  // COLOURED: the plan's part size, threads per block
};

// every knob any candidate sets, with the library's defaults
const Knobs kDefaults = {{"chain_persist", 0}, {"persist_et", 1024}, {"persist_u", 1},
                         {"persist_lag", -1},  {"fold_variant", 0},  {"flux_ctas_per_sm", 16},
                         {"chain_tiled", 0},   {"tile_threads", 1024}};

std::vector<Candidate> candidates(bool allow_reorder) {
  std::vector<Candidate> out;
  for (int fv : {0, 4, 5})
    for (int fc : {8, 16}) {
      Candidate c;
      c.knobs = {{"chain_persist", 0}, {"fold_variant", fv}, {"flux_ctas_per_sm", fc}};
      out.push_back(c);
    }
  for (int et : {512, 1024, 2048, 4096})
    for (int u : {1, 2})
      for (int lag : {-1, 16, 64, 256}) {
        Candidate c;
        c.knobs = {{"chain_persist", 1}, {"persist_et", et}, {"persist_u", u},
                   {"persist_lag", lag}};
        out.push_back(c);
      }
  for (int th : {1024, 512}) {  // the tiled one-launch chain
    Candidate c;
    c.knobs = {{"chain_tiled", 1}, {"tile_threads", th}};
    out.push_back(c);
  }
  if (allow_reorder)  // part size and threads per block of the colouring scheme
    for (auto pb : {std::make_pair(512, 512), std::make_pair(512, 256), std::make_pair(256, 256),
                    std::make_pair(256, 128), std::make_pair(128, 128), std::make_pair(64, 64)}) {
      Candidate c;
      c.strategy = OP2B_STRATEGY_COLOURED;
      c.part_size = pb.first;
      c.block_size = pb.second;
      out.push_back(c);
    }
  return out;
}

std::string describe(const Candidate &c) {
  std::string s;
  if (c.strategy == OP2B_STRATEGY_COLOURED)
    return "strategy=coloured,part_size=" + std::to_string(c.part_size) +
           ",block_size=" + std::to_string(c.block_size);
  for (auto &kv : c.knobs) {
    if (!s.empty()) s += ",";
    s += kv.first + "=" + std::to_string(kv.second);
  }
  return s;
}

// "key=value,key=value" back into a candidate; false on a malformed line
bool parse(const std::string &text, Candidate *c) {
  c->knobs.clear();
  c->strategy = OP2B_STRATEGY_GATHER;
  c->part_size = c->block_size = 0;
  size_t pos = 0;
  while (pos < text.size()) {
    size_t end = text.find(',', pos);
    if (end == std::string::npos) end = text.size();
    const std::string item = text.substr(pos, end - pos);
    const size_t eq = item.find('=');
    if (eq == std::string::npos || eq == 0) return false;
    const std::string k = item.substr(0, eq), v = item.substr(eq + 1);
    if (k == "strategy") {
      if (v != "coloured") return false;
      c->strategy = OP2B_STRATEGY_COLOURED;
    } else {
      char *e = nullptr;
      const long x = strtol(v.c_str(), &e, 10);
      if (!e || *e) return false;
      if (k == "part_size") c->part_size = (int)x;
      else if (k == "block_size") c->block_size = (int)x;
      else c->knobs.emplace_back(k, (int)x);
    }
    pos = end + 1;
  }
  return true;
}

// cache key of a chain: device, bytes per real, the four sets' sizes
std::string cache_key(const ChainArgs &c) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s|s%d|%d|%d|%d|%d", rt().device_name.c_str(),
           c.ra[2].dat->size / c.ra[2].dat->dim, c.rset->size, c.bset->size, c.uset->size,
           c.aa[0].dat->set->size);
  std::string k = buf;
  for (char &ch : k)
    if (ch == '\t' || ch == '\n') ch = ' ';
  return k;
}

void apply(const Candidate &c) {
  for (auto &kv : kDefaults) rt().tuning[kv.first] = kv.second;
  for (auto &kv : c.knobs) rt().tuning[kv.first] = kv.second;
  rt().strategy = c.strategy;
  if (c.strategy == OP2B_STRATEGY_COLOURED) {
    OP_part_size = c.part_size;
    if (c.block_size > 0) OP_block_size = c.block_size;
  }
}

}  // namespace
}  // namespace op2b

namespace op2b {
namespace {

// one launch of the chain as the dispatcher runs it with reductions
// deferred (GATHER: flux and fold, or the persistent launch) or loop by loop
// (COLOURED); the reductions are left undelivered.  false: not applicable
bool run_once(const ChainArgs &c, const Candidate &cand) {
  if (cand.strategy == OP2B_STRATEGY_COLOURED) {
    run_res_calc("res_calc", c.rset, c.ra.data());
    run_bres_calc("bres_calc", c.bset, c.ba.data());
    run_airfoil_update("update", c.uset, c.ua.data());
    run_adt_calc("adt_calc", c.aset, c.aa.data());
    return !error_pending();
  }
  std::vector<GblRequest> held;
  const bool ok = run_res_chain(nullptr, c.rset, c.ra.data(), c.bset, c.ba.data(), c.ua.data(),
                                c.aa.data(), nullptr, nullptr, nullptr, false, &held);
  return ok && !error_pending();
}

struct Snapshot {  // device copies of the datasets the chain writes
  std::vector<std::pair<op_dat, void *>> saved;
  bool take(const std::vector<op_dat> &dats) {
    for (op_dat d : dats) {
      bool dup = false;
      for (auto &s : saved) dup = dup || s.first == d;
      if (dup) continue;
      const size_t bytes = (size_t)d->size * d->set->size;
      void *p = dev_alloc(bytes);
      if (!p) return false;
      OP2B_CUDA(cudaMemcpyAsync(p, d->data_d, bytes, cudaMemcpyDeviceToDevice, rt().stream));
      saved.emplace_back(d, p);
    }
    return true;
  }
  void restore() {
    for (auto &s : saved)
      OP2B_CUDA(cudaMemcpyAsync(s.first->data_d, s.second, (size_t)s.first->size * s.first->set->size,
                                cudaMemcpyDeviceToDevice, rt().stream));
  }
  ~Snapshot() {
    cudaStreamSynchronize(rt().stream);
    for (auto &s : saved) dev_free(s.second);
  }
};

// mean device time of one chain launch (each after an L2 flush), or a
// negative value when the candidate does not apply
double time_candidate(const ChainArgs &c, const Candidate &cand, Snapshot &snap, int iters) {
  apply(cand);
  snap.restore();
  if (!run_once(c, cand)) return -1.0;  // untimed: builds plans and queues
  snap.restore();
  cudaStream_t s = rt().stream;
  std::vector<cudaEvent_t> ev(2 * iters);
  for (auto &e : ev) OP2B_CUDA(cudaEventCreate(&e));
  bool ok = true;
  for (int i = 0; i < iters && ok; i++) {
    op2b_l2_flush();
    OP2B_CUDA(cudaEventRecord(ev[2 * i], s));
    ok = run_once(c, cand);
    OP2B_CUDA(cudaEventRecord(ev[2 * i + 1], s));
  }
  OP2B_CUDA(cudaStreamSynchronize(s));
  double total = 0.0;
  for (int i = 0; i < iters && ok; i++) {
    float ms = 0.f;
    OP2B_CUDA(cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]));
    total += ms;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  return ok && !error_pending() ? 1e3 * total / iters : -1.0;
}

}  // namespace
}  // namespace op2b

using namespace op2b;

extern "C" int op2b_autotune(const char *cache_path, int iters, int allow_reorder) {
  flush_pending();
  if (error_pending()) return -1;
  ensure_cuda();
  if (live_graphs() > 0) {
    fail(-1, "op2b_autotune error: destroy the captured graphs first (they hold launch shapes)\n");
    return -1;
  }
  ChainArgs c;
  if (!last_res_chain(&c)) {
    fail(-1, "op2b_autotune error: no airfoil res_calc, bres_calc, update, adt_calc sequence "
             "has run yet; run one outer iteration first\n");
    return -1;
  }
  ahead_drop();  // nothing run ahead is swapped in after the trials
  // the trials leave the datasets as they found them, not as their flags say
  struct ForgetZeros {
    ~ForgetZeros() { known_zero_forget(); }
  } forget_zeros;
  alignas(16) static char gbl_scratch[16];  // the update's rms: never the caller's variable
  c.ua[4].data = gbl_scratch;
  const std::string key = cache_key(c);
  // 1. a cached choice for this device and mesh
  if (cache_path) {
    if (FILE *f = fopen(cache_path, "r")) {
      char line[1024];
      Candidate hit;
      bool found = false;
      while (fgets(line, sizeof line, f)) {
        std::string l = line;
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
        const size_t t1 = l.find('\t'), t2 = l.find('\t', t1 == std::string::npos ? 0 : t1 + 1);
        if (t1 == std::string::npos || t2 == std::string::npos) continue;
        Candidate cand;
        if (l.substr(0, t1) == key && parse(l.substr(t1 + 1, t2 - t1 - 1), &cand)) {
          hit = cand;  // the last entry for the key wins
          found = true;
        }
      }
      fclose(f);
      if (found) {
        apply(hit);
        return 1;
      }
    }
  }
  // 2. time every candidate on the app's data, putting the data back after each
  if (iters < 1) iters = 3;
  const int old_strategy = rt().strategy, old_part = OP_part_size, old_block = OP_block_size,
            old_mode = rt().error_mode;
  std::vector<std::pair<std::string, int>> old_knobs;
  for (auto &kv : kDefaults) old_knobs.emplace_back(kv.first, tuning(kv.first.c_str(), kv.second));
  Snapshot snap;
  if (!snap.take({c.ua[1].dat, c.ua[2].dat, c.ua[3].dat, c.aa[5].dat})) return -1;
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  rt().error_mode = OP2B_ERRORS_RETURN;  // a failing candidate is skipped, not fatal
  std::vector<Candidate> cands = candidates(allow_reorder != 0);
  int best = -1;
  double best_us = 0.0;
  for (size_t i = 0; i < cands.size(); i++) {
    const double us = time_candidate(c, cands[i], snap, iters);
    if (error_pending()) op2b_clear_error();
    if (us > 0.0 && (best < 0 || us < best_us)) {
      best = (int)i;
      best_us = us;
    }
  }
  rt().error_mode = old_mode;
  snap.restore();
  if (best < 0) {
    for (auto &kv : old_knobs) rt().tuning[kv.first] = kv.second;
    rt().strategy = old_strategy;
    OP_part_size = old_part;
    OP_block_size = old_block;
    fail(-1, "op2b_autotune error: no candidate launch shape ran\n");
    return -1;
  }
  OP_part_size = old_part;  // a COLOURED winner sets its own
  OP_block_size = old_block;
  apply(cands[best]);
  if (cache_path) {
    if (FILE *f = fopen(cache_path, "a")) {
      fprintf(f, "%s\t%s\t%.3f\n", key.c_str(), describe(cands[best]).c_str(), best_us);
      fclose(f);
    }
  }
  return 0;
}

extern "C" int op2b_get_tuning(const char *key, int def) { return key ? tuning(key, def) : def; }
