// device.cu -- device set-up and data movement: op_init, op_decl_dat_char,
// op_decl_const_char, op_fetch_data, op_exit (the CUDA half of the
// reference's common/op_lib.cu:82-209), the library stream and loop timers.
//
// Layout in HBM: each op_dat lives in one allocation in the app's own
// element-major order (element e, component d at e*dim+d).  Components of one
// element are contiguous, so a thread reads a whole element with one
// 8/16-byte vector load (float2 x, float4 q, 2 x double2 for FP64 q); the
// direct loops stream 16-byte vectors per thread, which coalesces fully.

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <unordered_set>
#include <vector>

#include "internal.h"

void op2b_release_plans();  // plan.cu

namespace op2b {

void release_fused_plans();  // airfoil.cu
void release_jac_pairs();    // jac.cu
void release_jac_steps();    // jac.cu

// bytes copied host -> device by dataset declarations and map uploads
static unsigned long long g_h2d_bytes = 0;

void ensure_cuda() {
  Runtime &R = rt();
  if (R.cuda_ready) return;
  int n = 0;
  cudaError_t err = cudaGetDeviceCount(&n);
  if (err != cudaSuccess || n == 0) {
    fail(-1, "op2b error: no CUDA device available (%s)\n",
         err == cudaSuccess ? "0 devices" : cudaGetErrorString(err));
    return;
  }
  // Host waits spin rather than yield: the drop-in API returns every global
  // reduction to the caller before the loop call returns, so each update is
  // a host round trip and its wake-up latency is GPU idle time.  This is a
  // flag of this process's context (set before it exists; ignored if the
  // process created it already); OP2B_SYNC_YIELD=1 keeps the default.
  const char *yield = getenv("OP2B_SYNC_YIELD");
  if (!(yield && yield[0] == '1') &&
      cudaSetDeviceFlags(cudaDeviceScheduleSpin | cudaDeviceMapHost) != cudaSuccess)
    cudaGetLastError();
  OP2B_CUDA(cudaGetDevice(&R.device));
  cudaDeviceProp prop;
  OP2B_CUDA(cudaGetDeviceProperties(&prop, R.device));
  R.num_sms = prop.multiProcessorCount;
  R.smem_optin = (int)prop.sharedMemPerBlockOptin;
  R.device_name = prop.name;
  if (prop.major < 10)
    fail(-1, "op2b error: device %s is sm_%d%d; this library is built for sm_100a\n", prop.name,
         prop.major, prop.minor);
  if (!R.stream) {
    OP2B_CUDA(cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking));
    R.own_stream = true;
  }
  R.cuda_ready = true;
}

// The library's long-lived device buffers (datasets, maps, plans, scratch)
// come from a private stream-ordered memory pool that keeps what is freed
// for reuse until the process exits (release threshold unbounded): on this
// pool's B200s cudaMalloc takes about 0.4 ms and cudaFree 0.3 ms, a pool
// allocation about 4 us, and a solve makes some twenty of each (every
// dataset and map, each plan), so a second solve in a process starts about
// 10 ms sooner.  An allocation is made on the library stream, which is then
// synchronised, so the buffer is usable from any stream or copy at once; a
// free is ordered after the library stream's work.  During a stream capture
// (which must not record allocations) and with OP2B_POOL=0 the plain
// cudaMalloc / cudaFree are used.
namespace {
cudaMemPool_t g_pool = nullptr;
int g_pool_device = -1;
bool g_pool_off = false, g_pool_checked = false;
std::unordered_set<void *> g_pooled;  // live buffers that came from the pool

bool stream_capturing() {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(rt().stream, &st) != cudaSuccess) {
    cudaGetLastError();
    return true;  // unknown: take the plain path
  }
  return st != cudaStreamCaptureStatusNone;
}

cudaMemPool_t pool() {
  if (!g_pool_checked) {
    const char *e = getenv("OP2B_POOL");
    g_pool_off = e && e[0] == '0';
    g_pool_checked = true;
  }
  if (g_pool_off) return nullptr;
  Runtime &R = rt();
  if (g_pool && g_pool_device == R.device) return g_pool;
  cudaMemPoolProps props;
  memset(&props, 0, sizeof props);
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = R.device;
  cudaMemPool_t p = nullptr;
  if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
    cudaGetLastError();
    g_pool_off = true;
    return nullptr;
  }
  unsigned long long keep = ~0ull;
  cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
  g_pool = p;
  g_pool_device = R.device;
  return g_pool;
}
}  // namespace

// stream-ordered scratch (plan building, the group engine's solves) from
// the same pool: cudaMallocAsync's default pool hands freed memory back at
// once, so each allocation maps pages again
cudaError_t pool_malloc_async(void **p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t mp = pool();
  return mp ? cudaMallocFromPoolAsync(p, bytes, mp, s) : cudaMallocAsync(p, bytes, s);
}

void *dev_alloc(size_t bytes) {
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  ensure_cuda();
  Runtime &R = rt();
  cudaMemPool_t mp = stream_capturing() ? nullptr : pool();
  cudaError_t err;
  if (mp) {
    err = cudaMallocFromPoolAsync(&p, bytes, mp, R.stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(R.stream);
    if (err == cudaSuccess) g_pooled.insert(p);
  } else {
    err = cudaMalloc(&p, bytes);
  }
  if (err != cudaSuccess) {
    fail(-1, "op2b error: allocation of %zu bytes failed: %s\n", bytes, cudaGetErrorString(err));
    return nullptr;
  }
  return p;
}

void dev_free(void *p) {
  if (!p) return;
  // pool memory goes back to the pool once the library stream's work is done
  auto it = g_pooled.find(p);
  if (it != g_pooled.end()) {
    g_pooled.erase(it);
    if (!stream_capturing()) {
      cudaFreeAsync(p, rt().stream);
      return;
    }
  }
  cudaFree(p);
}

// A map's device copy started at its declaration, so the copy runs while
// the host checks the map's entries and declares the rest: the upload is
// queued on the library stream (pool memory, no host wait), and a loop's
// first use of the map finds it there.  Not while renumbering is on (the
// copy would be rewritten anyway) or before CUDA is up.
void *map_upload_begin(const int *imap, size_t bytes) {
  Runtime &R = rt();
  if (!R.cuda_ready || renumber_enabled() || error_pending() || !imap || bytes == 0)
    return nullptr;
  if (stream_capturing()) return nullptr;
  void *d = nullptr;
  if (pool_malloc_async(&d, bytes, R.stream) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (cudaMemcpyAsync(d, imap, bytes, cudaMemcpyHostToDevice, R.stream) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(d, R.stream);
    return nullptr;
  }
  g_h2d_bytes += bytes;
  return d;
}

void map_upload_attach(op_map m, void *d) {
  if (!d) return;
  Runtime &R = rt();
  if (R.maps.size() <= (size_t)m->index) R.maps.resize(m->index + 1);
  MapDev &md = R.maps[m->index];
  if (md.d) {  // cannot happen for a new map; keep the existing copy
    cudaFreeAsync(d, R.stream);
    return;
  }
  md.d = (int *)d;
  g_pooled.insert(d);  // freed with dev_free like the other pool buffers
}

void map_upload_abort(void *d) {
  if (d) cudaFreeAsync(d, rt().stream);
}

const int *map_dev(op_map m) {
  Runtime &R = rt();
  if (!m) return nullptr;
  if (R.maps.size() <= (size_t)m->index) R.maps.resize(m->index + 1);
  MapDev &md = R.maps[m->index];
  if (!md.d) {
    ensure_cuda();
    size_t bytes = sizeof(int) * (size_t)m->dim * m->from->size;
    md.d = (int *)dev_alloc(bytes);
    if (md.d) {
      OP2B_CUDA(cudaMemcpyAsync(md.d, (const int *)m->map, bytes, cudaMemcpyHostToDevice,
                                R.stream));
      g_h2d_bytes += bytes;
      OP2B_CUDA(cudaStreamSynchronize(R.stream));
      // renumbered sets: rows in the from-set's new order, values in the
      // to-set's new numbering, rewritten on the device
      renumber_map_device(m, md.d);
    }
  }
  return md.d;
}

// device copies of maps and every plan, rebuilt on next use
void release_plans_and_maps() {
  ::op2b_release_plans();
  release_fused_plans();
  release_jac_steps();
  release_jac_pairs();
  for (auto &m : rt().maps) {
    dev_free(m.d);
    m.d = nullptr;
  }
}

static bool capturing() {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (rt().stream) cudaStreamIsCapturing(rt().stream, &st);
  return st != cudaStreamCaptureStatusNone;
}

LoopScope::LoopScope(char const *name, double transfer, double transfer2) {
  Runtime &R = rt();
  LoopTimer &T = R.timers[name];
  if (T.kernel_index < 0) {
    T.name = name;
    T.kernel_index = (int)R.timers.size() - 1;
  }
  t = &T;
  T.count++;
  op_timing_realloc(T.kernel_index);
  op_kernel &k = OP_kernels[T.kernel_index];
  k.name = T.name.c_str();
  k.count += 1;
  k.transfer += (float)transfer;
  k.transfer2 += (float)transfer2;
  if (capturing()) {
    // inside a graph capture: bracket the loop with event nodes of its own
    // (profiled graphs), or record nothing
    if (!R.capture_profile) return;
    OP2B_CUDA(cudaEventCreate(&ev.first));
    OP2B_CUDA(cudaEventCreate(&ev.second));
    // "external" records become event-record nodes of the graph (a plain
    // record inside a capture only expresses a dependency)
    OP2B_CUDA(cudaEventRecordWithFlags(ev.first, R.stream, cudaEventRecordExternal));
    captured = true;
    return;
  }
  if (!R.timing) return;
  first = T.count == 1;
  if (R.timing == 1 && !first && (T.count - 1) % kTimingSample != 0) return;
  if (T.pending.size() > 512) flush_timers();
  if (T.free_pairs.empty()) {
    cudaEvent_t a, b;
    OP2B_CUDA(cudaEventCreate(&a));
    OP2B_CUDA(cudaEventCreate(&b));
    T.free_pairs.push_back({a, b});
  }
  ev = T.free_pairs.back();
  T.free_pairs.pop_back();
  OP2B_CUDA(cudaEventRecord(ev.first, R.stream));
}

LoopScope::~LoopScope() {
  if (!ev.first) return;
  if (captured) cudaEventRecordWithFlags(ev.second, rt().stream, cudaEventRecordExternal);
  else cudaEventRecord(ev.second, rt().stream);
  if (captured) rt().capture_events.push_back({t->name, ev.first, ev.second});
  else t->pending.push_back(LoopTimer::Timed{ev, first});
}

PhaseScope::PhaseScope(const std::string &name) : name_(name) {
  Runtime &R = rt();
  if (!R.capture_profile || !capturing()) return;
  OP2B_CUDA(cudaEventCreate(&a_));
  OP2B_CUDA(cudaEventCreate(&b_));
  OP2B_CUDA(cudaEventRecordWithFlags(a_, R.stream, cudaEventRecordExternal));
}

PhaseScope::~PhaseScope() {
  if (!a_) return;
  cudaEventRecordWithFlags(b_, rt().stream, cudaEventRecordExternal);
  rt().capture_events.push_back({name_, a_, b_});
}

void flush_timers() {
  Runtime &R = rt();
  for (auto &kv : R.timers) {
    LoopTimer &T = kv.second;
    if (T.pending.empty()) continue;
    for (auto &p : T.pending) {
      float ms = 0.f;
      if (cudaEventSynchronize(p.ev.second) == cudaSuccess &&
          cudaEventElapsedTime(&ms, p.ev.first, p.ev.second) == cudaSuccess) {
        if (p.first) {
          T.first_s = ms * 1e-3;
        } else {
          T.sampled_s += ms * 1e-3;
          T.sampled_n++;
        }
      }
      T.free_pairs.push_back(p.ev);
    }
    T.pending.clear();
    // every call after the first at the sampled mean
    const double rest = T.sampled_n ? T.sampled_s / T.sampled_n * (T.count - 1) : 0.0;
    T.seconds = T.first_s + rest;
    if (T.kernel_index >= 0 && T.kernel_index < OP_kern_max)
      OP_kernels[T.kernel_index].time = (float)T.seconds;
  }
}

int const_get_f32(char const *name, float *out, int n) {
  auto it = rt().consts.find(name);
  if (it == rt().consts.end()) return 0;
  const Runtime::Const &c = it->second;
  int k = c.dim < n ? c.dim : n;
  for (int i = 0; i < k; i++) {
    if (c.type == "double") out[i] = (float)((const double *)c.bytes.data())[i];
    else if (c.type == "float") out[i] = ((const float *)c.bytes.data())[i];
    else if (c.type == "int") out[i] = (float)((const int *)c.bytes.data())[i];
    else return 0;
  }
  return k;
}

int const_get_f64(char const *name, double *out, int n) {
  auto it = rt().consts.find(name);
  if (it == rt().consts.end()) return 0;
  const Runtime::Const &c = it->second;
  int k = c.dim < n ? c.dim : n;
  for (int i = 0; i < k; i++) {
    if (c.type == "double") out[i] = ((const double *)c.bytes.data())[i];
    else if (c.type == "float") out[i] = (double)((const float *)c.bytes.data())[i];
    else if (c.type == "int") out[i] = (double)((const int *)c.bytes.data())[i];
    else return 0;
  }
  return k;
}

}  // namespace op2b

using namespace op2b;

extern void op2b_release_plans();  // plan.cu

extern "C" {

// common/op_lib.cu:128-143
void op_init(int argc, char **argv, int diags) {
  op_init_core(argc, argv, diags);
  ensure_cuda();
  if (!rt().cuda_ready) return;
  printf("\n Using CUDA device: %s\n", rt().device_name.c_str());
}

// whether the host bytes [p, p + n) are all zero: the first 4 KB alone, then
// one pass split over up to 8 host threads (a zero-filled calloc'd array
// that was never touched maps the zero page as it is read, page by page,
// which the threads do in parallel)
static bool host_all_zero(const char *p, size_t n) {
  auto part = [p](size_t a, size_t b) {
    unsigned long long acc = 0;
    size_t i = a;
    for (; i < b && ((uintptr_t)(p + i) & 7); i++) acc |= (unsigned char)p[i];
    const unsigned long long *w = reinterpret_cast<const unsigned long long *>(p + i);
    const size_t nw = (b - i) / 8;
    for (size_t k = 0; k < nw; k++) acc |= w[k];
    for (i += 8 * nw; i < b; i++) acc |= (unsigned char)p[i];
    return acc == 0;
  };
  const size_t head = std::min(n, (size_t)4096);
  if (!part(0, head)) return false;
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t nt = hw < 2 ? 1 : std::min<size_t>(8, hw);
  const size_t chunk = (n - head + nt - 1) / nt;
  std::vector<char> zero(nt, 1);
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; t++)
    th.emplace_back([&, t] {
      zero[t] = part(std::min(n, head + t * chunk), std::min(n, head + (t + 1) * chunk));
    });
  zero[0] = part(head, std::min(n, head + chunk));
  bool all = zero[0] != 0;
  for (size_t t = 1; t < nt; t++) {
    th[t - 1].join();
    all = all && zero[t] != 0;
  }
  return all;
}

// common/op_lib.cu:145-153: registry entry + device copy (synchronous, so
// the caller may reuse its array on return).  A large array in pageable
// host memory that holds only zero bytes (an app's zero-initialised qold,
// adt, res) is not copied: the device buffer is cleared instead, which
// gives the same bytes without the pageable copy's page-by-page staging,
// and the dataset is known to hold zeros.
op_dat op_decl_dat_char(op_set set, int dim, char const *type, int size, char *data,
                        char const *name) {
  op_dat dat = op_decl_dat_core(set, dim, type, size, data, name);
  if (!dat) return nullptr;
  Runtime &R = rt();
  ensure_cuda();
  if (R.dats.size() <= (size_t)dat->index) R.dats.resize(dat->index + 1);
  size_t bytes = (size_t)dat->size * set->size;
  R.dats[dat->index].bytes = bytes;
  dat->data_d = (char *)dev_alloc(bytes);
  if (!dat->data_d) return dat;
  bool zero = data == nullptr;
  if (data && bytes >= ((size_t)1 << 20) && tuning("decl_zero_scan", 1)) {
    cudaPointerAttributes pa;
    const bool pageable =
        cudaPointerGetAttributes(&pa, data) == cudaSuccess && pa.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();
    zero = pageable && host_all_zero(data, bytes);
  }
  if (zero) {
    OP2B_CUDA(cudaMemsetAsync(dat->data_d, 0, bytes, R.stream));
  } else {
    OP2B_CUDA(cudaMemcpyAsync(dat->data_d, data, bytes, cudaMemcpyHostToDevice, R.stream));
    g_h2d_bytes += bytes;
  }
  OP2B_CUDA(cudaStreamSynchronize(R.stream));
  permute_dat_in_place(dat);  // when its set has been renumbered
  if (zero && !error_pending()) dat_set_known_zero(dat, true);
  return dat;
}

// airfoil/airfoil_kernels.cu:23-26 copied constants to __constant__ symbols
// by name; here they are kept by name and handed to the loops as kernel
// parameters (the parameter bank is constant memory too).  A later
// declaration of the same name replaces the earlier one (jac2/jac.cpp:137-140).
void op_decl_const_char(int dim, char const *type, int size, char *dat, char const *name) {
  flush_pending();
  ahead_drop();  // values run ahead used the old constants
  if (dim <= 0 || size <= 0 || dat == nullptr) {
    fail(-1, "op_decl_const error -- invalid constant %s\n", name ? name : "(null)");
    return;
  }
  Runtime::Const c;
  c.type = type ? type : "";
  c.dim = dim;
  c.size = size;
  c.bytes.assign(dat, dat + (size_t)dim * size);
  rt().consts[name] = c;
  rt().consts_version++;
}

// op_seq.h's unnamed op_decl_const(dim, type, ptr): the name is the
// expression the app wrote ("&gam", "qinf", "& alpha"), without the address
// operator, blanks and enclosing parentheses
void op2b_decl_const_named(int dim, char const *type, int size, char *dat, char const *expr) {
  std::string e = expr ? expr : "";
  std::string n;
  for (char ch : e)
    if (ch != ' ' && ch != '\t' && ch != '(' && ch != ')') n += ch;
  while (!n.empty() && n[0] == '&') n.erase(0, 1);
  if (n.empty()) {
    fail(-1, "op_decl_const error -- cannot name the constant passed as \"%s\"\n",
         expr ? expr : "(null)");
    return;
  }
  op_decl_const_char(dim, type, size, dat, n.c_str());
}

// common/op_lib.cu:116-121: device -> the caller's original array
void op_fetch_data(op_dat dat) {
  flush_pending();
  if (!dat || !dat->data_d) return;
  Runtime &R = rt();
  deliver_deferred();
  if (fetch_unpermuted(dat, dat->data)) return;  // renumbered set: the app's order back
  OP2B_CUDA(cudaMemcpyAsync(dat->data, dat->data_d, (size_t)dat->size * dat->set->size,
                            cudaMemcpyDeviceToHost, R.stream));
  OP2B_CUDA(cudaStreamSynchronize(R.stream));
}

// common/op_lib.cu:186-209
void op_exit(void) {
  flush_pending();
  Runtime &R = rt();
  if (R.cuda_ready) {
    deliver_deferred();
    cudaStreamSynchronize(R.stream);
    flush_timers();
  }
  op2b_release_plans();
  release_fused_plans();
  release_jac_steps();
  release_jac_pairs();
  renumber_reset();
  checkpoint_reset();
  ahead_reset();
  noalloc_reset();
  release_tile_alts();
  for (auto &m : R.maps) dev_free(m.d);
  R.maps.clear();
  for (int i = 0; i < OP_dat_index; i++) dev_free(OP_dat_list[i]->data_d);
  R.dats.clear();
  for (auto &kv : R.timers) {
    for (auto &p : kv.second.free_pairs) {
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
  }
  R.timers.clear();
  R.consts.clear();
  R.consts_version++;  // constants cached by the loops are stale now
  op_exit_core();
}

void *op2b_get_stream(void) {
  ensure_cuda();
  return (void *)rt().stream;
}

void op2b_set_stream(void *s) {
  ensure_cuda();
  Runtime &R = rt();
  if (R.stream && R.stream != (cudaStream_t)s) cudaStreamSynchronize(R.stream);
  R.stream = (cudaStream_t)s;
  R.own_stream = false;
}

int op2b_sync(void) {
  flush_pending();
  ensure_cuda();
  deliver_deferred();
  return (int)cudaStreamSynchronize(rt().stream);
}

double op2b_loop_time(char const *name, int *count) {
  flush_pending();
  flush_timers();
  auto it = rt().timers.find(name);
  if (it == rt().timers.end()) return -1.0;
  if (count) *count = it->second.count;
  return it->second.seconds;
}

}  // extern "C"

// Reads (never writes) a buffer three times the size of L2, so the next
// kernel starts with a cold cache and no dirty lines to write back.
static __global__ void k_l2_sweep(const uint4 *__restrict__ p, size_t n, unsigned *sink) {
  uint4 acc = make_uint4(0, 0, 0, 0);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint4 v = __ldcg(p + i);
    acc.x ^= v.x; acc.y ^= v.y; acc.z ^= v.z; acc.w ^= v.w;
  }
  if ((acc.x ^ acc.y ^ acc.z ^ acc.w) == 0x9e3779b9u) *sink = 1u;  // keeps the loads
}

extern "C" {

int op2b_l2_flush(void) {
  ensure_cuda();
  static void *buf = nullptr;
  static size_t bytes = 0;
  if (!buf) {
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, rt().device);
    bytes = (size_t)(l2 > 0 ? l2 : 128 << 20) * 3;
    buf = dev_alloc(bytes + 256);
    if (!buf) return (int)cudaErrorMemoryAllocation;
    OP2B_CUDA(cudaMemset(buf, 0, bytes + 256));
  }
  k_l2_sweep<<<rt().num_sms * 8, 256, 0, rt().stream>>>((const uint4 *)buf, bytes / 16,
                                                        (unsigned *)((char *)buf + bytes));
  return (int)cudaGetLastError();
}

unsigned long long op2b_h2d_bytes(int reset) {
  const unsigned long long n = op2b::g_h2d_bytes;
  if (reset) op2b::g_h2d_bytes = 0;
  return n;
}

char const *op2b_version(void) {
  return "libop2b200 (sm_100a; -fmad=false, IEEE div/sqrt)";
}

}  // extern "C"
