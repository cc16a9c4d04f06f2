// core.cpp -- registries, argument construction and checks, diagnostics and
// timing tables.  Host C++ with the C API of the reference's C99 core
// (common/op_lib_core.c:36-445); error messages and exit codes are the
// reference's, so apps and scripts that parse them keep working.

#include <stdarg.h>
#include <sys/time.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

extern "C" {
int OP_diags = 0, OP_part_size = 0, OP_block_size = 512, OP_cache_line_size = 128;
int OP_set_index = 0, OP_set_max = 0, OP_map_index = 0, OP_map_max = 0, OP_dat_index = 0,
    OP_dat_max = 0, OP_plan_index = 0, OP_plan_max = 0, OP_kern_max = 0;
op_set *OP_set_list = nullptr;
op_map *OP_map_list = nullptr;
op_dat *OP_dat_list = nullptr;
op_plan *OP_plans = nullptr;
op_kernel *OP_kernels = nullptr;
}

namespace op2b {

static thread_local std::string g_last_error;
static thread_local bool g_error_pending = false;

Runtime &rt() {
  static Runtime r;
  return r;
}

void fail(int exit_code, const char *fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  printf("%s", buf);
  fflush(stdout);
  if (rt().error_mode == OP2B_ERRORS_EXIT) exit(exit_code);
  g_last_error = buf;
  g_error_pending = true;
}

bool error_pending() { return g_error_pending; }

void cuda_fail(cudaError_t err, const char *what, const char *file, int line) {
  fail(-1, "%s(%i) : CUDA runtime error : %s (%s).\n", file, line, cudaGetErrorString(err), what);
}

// registries grow in steps of 10 entries (common/op_lib_core.c:102-109)
template <class T>
static bool grow(T **list, int index, int *max) {
  if (index < *max) return true;
  *max += 10;
  T *p = (T *)realloc(*list, (size_t)*max * sizeof(T));
  if (!p) return false;
  *list = p;
  return true;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

const char *op2b_last_error(void) { return g_last_error.c_str(); }
void op2b_clear_error(void) {
  g_last_error.clear();
  g_error_pending = false;
}
int op2b_set_error_mode(int mode) {
  int old = rt().error_mode;
  rt().error_mode = mode;
  return old;
}
int op2b_set_strategy(int s) {
  flush_pending();
  int old = rt().strategy;
  rt().strategy = s;
  return old;
}
int op2b_set_reduction(int m) {
  flush_pending();
  int old = rt().reduction;
  rt().reduction = m;
  return old;
}
int op2b_set_tuning(const char *key, int value) {
  flush_pending();
  if (!key) return -1;
  int old = tuning(key, -1);
  rt().tuning[key] = value;
  return old;
}

int op2b_set_timing(int mode) {
  int old = rt().timing;
  rt().timing = mode < 0 ? 0 : (mode > 2 ? 2 : mode);
  return old;
}

// common/op_lib_core.c:68-92
void op_init_core(int argc, char **argv, int diags) {
  OP_diags = diags;
#ifdef OP_BLOCK_SIZE
  OP_block_size = OP_BLOCK_SIZE;
#endif
#ifdef OP_PART_SIZE
  OP_part_size = OP_PART_SIZE;
#endif
  for (int n = 1; n < argc; n++) {
    if (strncmp(argv[n], "OP_BLOCK_SIZE=", 14) == 0) {
      OP_block_size = atoi(argv[n] + 14);
      printf("\n OP_block_size = %d \n", OP_block_size);
    }
    if (strncmp(argv[n], "OP_PART_SIZE=", 13) == 0) {
      OP_part_size = atoi(argv[n] + 13);
      printf("\n OP_part_size  = %d \n", OP_part_size);
    }
    if (strncmp(argv[n], "OP_CACHE_LINE_SIZE=", 19) == 0) {
      OP_cache_line_size = atoi(argv[n] + 19);
      printf("\n OP_cache_line_size  = %d \n", OP_cache_line_size);
    }
  }
}

// common/op_lib_core.c:94-119
op_set op_decl_set(int size, char const *name) {
  if (size <= 0) {
    fail(-1, " op_decl_set error -- negative/zero size for set: %s\n", name);
    return nullptr;
  }
  if (!grow(&OP_set_list, OP_set_index, &OP_set_max)) {
    fail(-1, " op_decl_set error -- error reallocating memory\n");
    return nullptr;
  }
  op_set set = (op_set)malloc(sizeof(op_set_core));
  set->index = OP_set_index;
  set->size = size;
  set->name = name;
  OP_set_list[OP_set_index++] = set;
  return set;
}

// common/op_lib_core.c:121-169
// 1 when some entry of imap[0, n) is outside [0, lim): one vectorisable
// pass, split over host threads for large maps (the check reads every entry
// of a multi-million-entry map; one thread streams it at about 15 GB/s)
static unsigned range_check(const int *imap, size_t n, unsigned lim) {
  auto part = [&](size_t a, size_t b) {
    unsigned bad = 0;
    for (size_t i = a; i < b; i++) bad |= (unsigned)((unsigned)imap[i] >= lim);
    return bad;
  };
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t nt = n < ((size_t)1 << 20) || hw < 2 ? 1 : std::min<size_t>(8, hw);
  if (nt == 1) return part(0, n);
  std::vector<unsigned> bad(nt, 0);
  std::vector<std::thread> th;
  const size_t chunk = (n + nt - 1) / nt;
  for (size_t t = 1; t < nt; t++)
    th.emplace_back([&, t] { bad[t] = part(std::min(n, t * chunk), std::min(n, (t + 1) * chunk)); });
  bad[0] = part(0, std::min(n, chunk));
  unsigned any = bad[0];
  for (size_t t = 1; t < nt; t++) {
    th[t - 1].join();
    any |= bad[t];
  }
  return any;
}

op_map op_decl_map(op_set from, op_set to, int dim, int *imap, char const *name) {
  if (from == nullptr) {
    fail(-1, " op_decl_map error -- invalid 'from' set for map %s\n", name);
    return nullptr;
  }
  if (to == nullptr) {
    fail(-1, "op_decl_map error -- invalid 'to' set for map %s\n", name);
    return nullptr;
  }
  if (dim <= 0) {
    fail(-1, "op_decl_map error -- negative/zero dimension for map %s\n", name);
    return nullptr;
  }
  // one contiguous, vectorisable pass decides whether any entry is out of
  // range; only then the reference's dimension-major scan finds the first
  // bad entry for the message
  const size_t nent = (size_t)dim * from->size;
  const unsigned lim = (unsigned)to->size;
  // the device copy (when the GPU is up) is queued first and runs during
  // the check
  void *dcopy = map_upload_begin(imap, sizeof(int) * nent);
  unsigned bad = range_check(imap, nent, lim);
  if (bad)
    for (int d = 0; d < dim; d++)
      for (int n = 0; n < from->size; n++) {
        int v = imap[d + (size_t)n * dim];
        if (v < 0 || v >= to->size) {
          map_upload_abort(dcopy);
          fail(-1,
               "op_decl_map error -- invalid data for map %s\n"
               "element = %d, dimension = %d, map = %d\n",
               name, n, d, v);
          return nullptr;
        }
      }
  if (!grow(&OP_map_list, OP_map_index, &OP_map_max)) {
    map_upload_abort(dcopy);
    fail(-1, " op_decl_map error -- error reallocating memory\n");
    return nullptr;
  }
  op_map map = (op_map)malloc(sizeof(op_map_core));
  map->index = OP_map_index;
  map->from = from;
  map->to = to;
  map->dim = dim;
  map->map = imap;
  map->name = name;
  OP_map_list[OP_map_index++] = map;
  // without a GPU (or with renumbering on) the device copy is made on first
  // use by a loop (map_dev), so declaring maps needs no GPU, as in the
  // reference
  map_upload_attach(map, dcopy);
  return map;
}

// common/op_lib_core.c:171-207
op_dat op_decl_dat_core(op_set set, int dim, char const *type, int size, char *data,
                        char const *name) {
  if (set == nullptr) {
    fail(-1, "op_decl_dat error -- invalid set for data: %s\n", name);
    return nullptr;
  }
  if (dim <= 0) {
    fail(-1, "op_decl_dat error -- negative/zero dimension for data: %s\n", name);
    return nullptr;
  }
  if (!grow(&OP_dat_list, OP_dat_index, &OP_dat_max)) {
    fail(-1, " op_decl_dat error -- error reallocating memory\n");
    return nullptr;
  }
  op_dat dat = (op_dat)malloc(sizeof(op_dat_core));
  dat->index = OP_dat_index;
  dat->set = set;
  dat->dim = dim;
  dat->data = data;
  dat->data_d = nullptr;
  dat->name = name;
  dat->type = type;
  dat->size = dim * size;
  OP_dat_list[OP_dat_index++] = dat;
  return dat;
}

// common/op_lib_core.c:209-254 (plans are released by op_exit first)
void op_exit_core(void) {
  free(OP_plans);
  OP_plans = nullptr;
  for (int i = 0; i < OP_set_index; i++) free(OP_set_list[i]);
  free(OP_set_list);
  for (int i = 0; i < OP_map_index; i++) free(OP_map_list[i]);
  free(OP_map_list);
  for (int i = 0; i < OP_dat_index; i++) free(OP_dat_list[i]);
  free(OP_dat_list);
  free(OP_kernels);
  OP_set_list = nullptr;
  OP_map_list = nullptr;
  OP_dat_list = nullptr;
  OP_kernels = nullptr;
  OP_set_index = OP_set_max = 0;
  OP_map_index = OP_map_max = 0;
  OP_dat_index = OP_dat_max = 0;
  OP_plan_index = OP_plan_max = 0;
  OP_kern_max = 0;
}

static void op_err_print(const char *error_string, int m, const char *name) {
  fail(1, "error: arg %d in kernel \"%s\"\n%s \n", m, name, error_string);
}

// common/op_lib_core.c:266-305
void op_arg_check(op_set set, int m, op_arg arg, int *ninds, char const *name) {
  if (arg.argtype == OP_ARG_DAT) {
    if (set == nullptr) return op_err_print("invalid set", m, name);
    if (arg.dat == nullptr) return op_err_print("invalid dataset", m, name);
    if (arg.map == nullptr && arg.dat->set != set)
      return op_err_print("dataset set does not match loop set", m, name);
    if (arg.map != nullptr && (arg.map->from != set || arg.map->to != arg.dat->set))
      return op_err_print("mapping error", m, name);
    if ((arg.map == nullptr && arg.idx != -1) ||
        (arg.map != nullptr && (arg.idx < 0 || arg.idx >= arg.map->dim)))
      return op_err_print("invalid index", m, name);
    if (arg.dat->dim != arg.dim)
      return op_err_print("dataset dim does not match declared dim", m, name);
    if (strcmp(arg.dat->type, arg.type))
      return op_err_print("dataset type does not match declared type", m, name);
    if (arg.idx >= 0) (*ninds)++;
  }
  if (arg.argtype == OP_ARG_GBL) {
    if (!strcmp(arg.type, "error"))
      return op_err_print("datatype does not match declared type", m, name);
    if (arg.dim <= 0) return op_err_print("dimension should be strictly positive", m, name);
    if (arg.data == nullptr) return op_err_print("NULL pointer for global data", m, name);
  }
}

// common/op_lib_core.c:307-326
op_arg op_arg_dat(op_dat dat, int idx, op_map map, int dim, char const *typ, op_access acc) {
  op_arg arg;
  memset(&arg, 0, sizeof arg);
  arg.argtype = OP_ARG_DAT;
  arg.dat = dat;
  arg.map = map;
  arg.dim = dim;
  arg.idx = idx;
  if (dat != nullptr) {
    arg.size = dat->size;
    arg.data = dat->data;
    arg.data_d = dat->data_d;
  }
  arg.type = typ;
  arg.acc = acc;
  return arg;
}

// common/op_lib_core.c:329-345
op_arg op_arg_gbl_core(char *data, int dim, char const *typ, op_access acc) {
  op_arg arg;
  memset(&arg, 0, sizeof arg);
  arg.argtype = OP_ARG_GBL;
  arg.dat = nullptr;
  arg.map = nullptr;
  arg.dim = dim;
  arg.idx = -1;
  arg.size = 0;
  arg.data = data;
  arg.type = typ;
  arg.acc = acc;
  return arg;
}

// common/op_lib_core.c:351-379
void op_diagnostic_output(void) {
  if (OP_diags > 1) {
    printf("\n  OP diagnostic output\n");
    printf("  --------------------\n");
    printf("\n       set       size\n");
    printf("  -------------------\n");
    for (int n = 0; n < OP_set_index; n++)
      printf("%10s %10d\n", OP_set_list[n]->name, OP_set_list[n]->size);
    printf("\n       map        dim       from         to\n");
    printf("  -----------------------------------------\n");
    for (int n = 0; n < OP_map_index; n++)
      printf("%10s %10d %10s %10s\n", OP_map_list[n]->name, OP_map_list[n]->dim,
             OP_map_list[n]->from->name, OP_map_list[n]->to->name);
    printf("\n       dat        dim        set\n");
    printf("  ------------------------------\n");
    for (int n = 0; n < OP_dat_index; n++)
      printf("%10s %10d %10s\n", OP_dat_list[n]->name, OP_dat_list[n]->dim,
             OP_dat_list[n]->set->name);
    printf("\n");
  }
}

// common/op_lib_core.c:381-403; "time" is summed device time of the loop's
// kernels (CUDA events) rather than host wall time around a synchronising
// stub, because loops here do not synchronise.
void op_timing_output(void) {
  flush_pending();
  flush_timers();
  if (OP_kern_max > 0) {
    printf("\n  count     time     GB/s     GB/s   kernel name ");
    printf("\n ----------------------------------------------- \n");
    for (int n = 0; n < OP_kern_max; n++) {
      op_kernel &k = OP_kernels[n];
      if (k.count > 0) {
        if (k.transfer2 == 0.0f)
          printf(" %6d  %8.4f %8.4f            %s \n", k.count, k.time,
                 k.transfer / (1e9f * k.time), k.name);
        else
          printf(" %6d  %8.4f %8.4f %8.4f   %s \n", k.count, k.time,
                 k.transfer / (1e9f * k.time), k.transfer2 / (1e9f * k.time), k.name);
      }
    }
  }
}

// common/op_lib_core.c:405-431
void op_timing_realloc(int kernel) {
  if (kernel >= OP_kern_max) {
    int nmax = kernel + 10;
    op_kernel *p = (op_kernel *)realloc(OP_kernels, (size_t)nmax * sizeof(op_kernel));
    if (!p) {
      fail(-1, " op_timing_realloc error \n");
      return;
    }
    OP_kernels = p;
    for (int n = OP_kern_max; n < nmax; n++) {
      OP_kernels[n].count = 0;
      OP_kernels[n].time = 0.0f;
      OP_kernels[n].transfer = 0.0f;
      OP_kernels[n].transfer2 = 0.0f;
      OP_kernels[n].name = "unused";
    }
    OP_kern_max = nmax;
  }
}

// common/op_lib_core.c:440-445
void op_timers(double *cpu, double *et) {
  (void)cpu;
  struct timeval t;
  gettimeofday(&t, nullptr);
  *et = t.tv_sec + t.tv_usec * 1.0e-6;
}

}  // extern "C"
