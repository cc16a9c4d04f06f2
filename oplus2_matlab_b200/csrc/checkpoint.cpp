// checkpoint.cpp -- op_checkpoint: save and fast-forward restart, as the
// reference's developer notes propose it (doc/dev.tex:1080-1087): a
// checkpoint saves every dataset and every global reduction value OP2 has
// returned to the app; a restarted app runs from the beginning in
// "fast-forward" -- its loop calls do not run, they hand back the recorded
// reduction values, which is all the app's control flow sees of OP2 -- and
// at the checkpoint the datasets are restored and execution continues.
//
// File (written to path.tmp, then renamed): "OP2BCKP1", the number of loop
// calls before the checkpoint, the number of checkpoint calls before it, the
// log of returned reduction values (per loop call: call number, argument
// number, bytes), then every dataset by name, set size, element size and
// bytes in the app's element order.
//
// Requires reductions delivered at each loop call (not op2b_set_gbl_deferred)
// and no graph capture while logging.  During fast-forward, op_fetch_data
// leaves host arrays as they are (the datasets do not exist yet).

#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "internal.h"

namespace op2b {
namespace {

struct GblRecord {
  long long call;
  int arg;
  std::vector<char> bytes;
};

struct DatRecord {
  std::string name;
  int set_size = 0, size = 0;
  std::vector<char> bytes;
};

struct Ckpt {
  std::string path;
  long long calls = 0;        // loop calls so far (this run)
  long long ckpt_calls = 0;   // op_checkpoint calls so far
  std::vector<GblRecord> log;  // reduction values returned so far
  // fast-forward state, from the file
  bool ff = false;
  long long ff_calls = 0, ff_ckpt = 0;
  std::vector<GblRecord> ff_log;
  size_t ff_next = 0;
  std::vector<DatRecord> ff_dats;
};

Ckpt &ck() {
  static Ckpt c;
  return c;
}

int type_bytes(const char *t) {
  if (!t) return 0;
  if (!strcmp(t, "double")) return 8;
  if (!strcmp(t, "float") || !strcmp(t, "int")) return 4;
  return 0;
}

bool wr(FILE *f, const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }
bool rd(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

bool load(const std::string &path, Ckpt &c) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[8];
  long long calls = 0, nck = 0, nlog = 0, ndat = 0;
  bool ok = rd(f, magic, 8) && !memcmp(magic, "OP2BCKP1", 8) && rd(f, &calls, 8) &&
            rd(f, &nck, 8) && rd(f, &nlog, 8);
  std::vector<GblRecord> log;
  for (long long i = 0; ok && i < nlog; i++) {
    GblRecord r;
    int n = 0;
    ok = rd(f, &r.call, 8) && rd(f, &r.arg, 4) && rd(f, &n, 4) && n >= 0 && n <= 4096;
    if (ok) {
      r.bytes.resize(n);
      ok = rd(f, r.bytes.data(), n);
    }
    log.push_back(std::move(r));
  }
  ok = ok && rd(f, &ndat, 8);
  std::vector<DatRecord> dats;
  for (long long i = 0; ok && i < ndat; i++) {
    DatRecord d;
    int nl = 0;
    long long nb = 0;
    ok = rd(f, &nl, 4) && nl > 0 && nl < 4096;
    if (ok) {
      d.name.resize(nl);
      ok = rd(f, &d.name[0], nl) && rd(f, &d.set_size, 4) && rd(f, &d.size, 4) && rd(f, &nb, 8) &&
           nb == (long long)d.set_size * d.size;
    }
    if (ok) {
      d.bytes.resize((size_t)nb);
      ok = rd(f, d.bytes.data(), (size_t)nb);
    }
    dats.push_back(std::move(d));
  }
  fclose(f);
  if (!ok) return false;
  c.ff_calls = calls;
  c.ff_ckpt = nck;
  c.ff_log = std::move(log);
  c.ff_dats = std::move(dats);
  c.ff_next = 0;
  return true;
}

// restore every dataset recorded in the file (matched by name and shape)
void restore(Ckpt &c) {
  ahead_drop();  // the datasets change under anything run ahead
  known_zero_forget();
  if (renumber_enabled()) renumber_apply();
  int found = 0;
  for (const DatRecord &r : c.ff_dats)
    for (int k = 0; k < OP_dat_index; k++) {
      op_dat d = OP_dat_list[k];
      if (!d->name || r.name != d->name || d->set->size != r.set_size || d->size != r.size ||
          !d->data_d)
        continue;
      OP2B_CUDA(cudaMemcpyAsync(d->data_d, r.bytes.data(), r.bytes.size(), cudaMemcpyHostToDevice,
                                rt().stream));
      OP2B_CUDA(cudaStreamSynchronize(rt().stream));
      permute_dat_in_place(d);
      found++;
      break;
    }
  if (found != (int)c.ff_dats.size())
    fail(-1, "op_checkpoint error -- %d of %d saved datasets have no match in this run\n",
         (int)c.ff_dats.size() - found, (int)c.ff_dats.size());
  c.ff = false;
  c.ff_dats.clear();
  c.ff_log.clear();
}

}  // namespace

// op2b_par_loop, before running a call: true = fast-forwarded (skip it)
bool checkpoint_before_loop(char const *name, int nargs, const op_arg *args) {
  Ckpt &c = ck();
  if (!c.ff) return false;
  const long long call = c.calls + 1;
  if (call > c.ff_calls) {
    fail(-1, "op_checkpoint error -- loop \"%s\" reached before the checkpoint it resumes\n",
         name);
    c.ff = false;
    return false;
  }
  c.calls = call;
  // hand back the values this call returned in the saved run
  while (c.ff_next < c.ff_log.size() && c.ff_log[c.ff_next].call == call) {
    const GblRecord &r = c.ff_log[c.ff_next++];
    if (r.arg < 0 || r.arg >= nargs || args[r.arg].argtype != OP_ARG_GBL || !args[r.arg].data) {
      fail(-1, "op_checkpoint error -- loop \"%s\" does not match the saved run\n", name);
      return true;
    }
    memcpy(args[r.arg].data, r.bytes.data(), r.bytes.size());
    c.log.push_back(r);
  }
  return true;
}

// op2b_par_loop, after a call has run and delivered its reductions
void checkpoint_after_loop(int nargs, const op_arg *args) {
  Ckpt &c = ck();
  if (c.path.empty()) return;
  c.calls++;
  for (int m = 0; m < nargs; m++) {
    const op_arg &a = args[m];
    if (a.argtype != OP_ARG_GBL || a.acc == OP_READ || !a.data) continue;
    const int n = a.dim * type_bytes(a.type);
    if (n <= 0) continue;
    c.log.push_back(GblRecord{c.calls, m, std::vector<char>(a.data, a.data + n)});
  }
}

bool checkpoint_fast_forward() { return ck().ff; }

void checkpoint_reset() { ck() = Ckpt(); }

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_checkpoint_file(const char *path) {
  Ckpt &c = ck();
  c = Ckpt();
  if (!path || !path[0]) return 0;
  c.path = path;
  if (load(c.path, c)) {
    c.ff = true;
    return 1;  // a checkpoint to resume from
  }
  return 0;
}

int op_checkpoint(void) {
  Ckpt &c = ck();
  if (c.path.empty()) {
    fail(-1, "op_checkpoint error -- no checkpoint file (op2b_checkpoint_file)\n");
    return -1;
  }
  c.ckpt_calls++;
  if (c.ff) {
    if (c.ckpt_calls < c.ff_ckpt) return 0;  // an earlier checkpoint of the saved run
    if (c.calls != c.ff_calls) {
      fail(-1, "op_checkpoint error -- the run does not match the saved one\n");
      return -1;
    }
    restore(c);
    return error_pending() ? -1 : 2;  // resumed here
  }
  flush_pending();
  if (rt().gbl_deferred) {
    fail(-1, "op_checkpoint error -- deferred global reductions are not logged\n");
    return -1;
  }
  if (rt().cuda_ready) OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  std::string tmp = c.path + ".tmp";
  FILE *f = fopen(tmp.c_str(), "wb");
  if (!f) {
    fail(-1, "op_checkpoint error -- cannot write %s\n", tmp.c_str());
    return -1;
  }
  long long nlog = (long long)c.log.size(), ndat = 0;
  for (int k = 0; k < OP_dat_index; k++)
    if (OP_dat_list[k]->data_d && OP_dat_list[k]->name) ndat++;
  bool ok = wr(f, "OP2BCKP1", 8) && wr(f, &c.calls, 8) && wr(f, &c.ckpt_calls, 8) &&
            wr(f, &nlog, 8);
  for (const GblRecord &r : c.log) {
    const int n = (int)r.bytes.size();
    ok = ok && wr(f, &r.call, 8) && wr(f, &r.arg, 4) && wr(f, &n, 4) && wr(f, r.bytes.data(), n);
  }
  ok = ok && wr(f, &ndat, 8);
  std::vector<char> buf;
  for (int k = 0; ok && k < OP_dat_index; k++) {
    op_dat d = OP_dat_list[k];
    if (!d->data_d || !d->name) continue;
    const int nl = (int)strlen(d->name);
    const long long nb = (long long)d->set->size * d->size;
    buf.resize((size_t)nb);
    if (!fetch_unpermuted(d, buf.data())) {
      OP2B_CUDA(cudaMemcpyAsync(buf.data(), d->data_d, (size_t)nb, cudaMemcpyDeviceToHost,
                                rt().stream));
      OP2B_CUDA(cudaStreamSynchronize(rt().stream));
    }
    ok = wr(f, &nl, 4) && wr(f, d->name, nl) && wr(f, &d->set->size, 4) && wr(f, &d->size, 4) &&
         wr(f, &nb, 8) && wr(f, buf.data(), (size_t)nb);
  }
  ok = (fclose(f) == 0) && ok;
  if (!ok || rename(tmp.c_str(), c.path.c_str()) != 0) {
    remove(tmp.c_str());
    fail(-1, "op_checkpoint error -- writing %s failed\n", c.path.c_str());
    return -1;
  }
  return 1;
}

}  // extern "C"
