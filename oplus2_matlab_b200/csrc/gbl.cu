// gbl.cu -- host side of global reductions: device scratch, result slots,
// and delivery into the caller's variables.
//
// Semantics kept from the reference CUDA back-end (airfoil/update_kernel.cu:
// 116-169, jac1/update_kernel.cu:94-141): OP_INC adds the device sum to the
// host value, OP_MAX / OP_MIN combine with it; the variable holds the result
// when the loop call returns.  In deferred mode the device results wait in
// slots until op2b_sync / op_fetch_data, so no call blocks.

#include <string.h>

#include <algorithm>

#include "loops.h"

namespace op2b {

namespace {
constexpr int kSlots = 4096;
struct RedState {
  char *dev = nullptr;  // [2 x kMaxRedBlocks x 8] partials | ticket (256 B)
  // result slots in mapped pinned host memory: the last block of a reduction
  // stores the result where the host reads it, so delivery needs no copy
  char *host = nullptr;
  int next_slot = 0;
  int graph_slots = 0;  // slots baked into captured graphs stay reserved
  void *seq = nullptr;
  size_t seq_bytes = 0;
};
RedState &rs() {
  static RedState s;
  return s;
}
size_t off_ticket() { return 2 * (size_t)kMaxRedBlocks * 8; }
size_t off_slots() { return off_ticket() + 256; }

void ensure_red() {
  RedState &S = rs();
  if (S.dev) return;
  size_t bytes = off_slots();
  S.dev = (char *)dev_alloc(bytes);
  OP2B_CUDA(cudaMemset(S.dev, 0, bytes));
  OP2B_CUDA(cudaHostAlloc((void **)&S.host, (size_t)kSlots * 8, cudaHostAllocMapped));
  memset(S.host, 0, (size_t)kSlots * 8);
}

template <class T>
void combine(char *host, const T v, op_access acc, bool assign) {
  T *h = (T *)host;
  switch (acc) {
    case OP_INC: *h = assign ? v : (T)(*h + v); break;
    case OP_MAX: *h = (*h > v) ? *h : v; break;
    case OP_MIN: *h = (*h < v) ? *h : v; break;
    default: break;
  }
}

void deliver(const std::vector<GblRequest> &reqs) {
  RedState &S = rs();
  if (reqs.empty()) return;
  int lo = kSlots, hi = -1;
  for (auto &r : reqs) {
    lo = std::min(lo, r.slot);
    hi = std::max(hi, r.slot);
  }
  (void)lo;
  (void)hi;
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));  // the slots are host memory
  for (auto &r : reqs) {
    const char *p = S.host + (size_t)r.slot * 8;
    if (r.type == GBL_F64) combine<double>(r.host, *(const double *)p, r.acc, r.assign);
    else combine<float>(r.host, *(const float *)p, r.acc, r.assign);
  }
}

std::vector<GblRequest> &pending() {
  static std::vector<GblRequest> v;
  return v;
}
}  // namespace

void *red_partials(int i) {
  ensure_red();
  return rs().dev + (size_t)i * kMaxRedBlocks * 8;
}

unsigned *red_ticket() {
  ensure_red();
  return (unsigned *)(rs().dev + off_ticket());
}

void *red_slot_ptr(int slot) {
  ensure_red();
  return rs().host + (size_t)slot * 8;  // a mapped host address (unified addressing)
}

int red_new_slot() {
  ensure_red();
  RedState &S = rs();
  if (S.next_slot >= kSlots) {
    deliver_deferred();  // frees every slot not held by a captured graph
    S.next_slot = S.graph_slots ? S.graph_slots : 0;
    if (S.next_slot >= kSlots) {
      fail(-1, "op2b error: global reduction slots exhausted by captured graphs\n");
      S.next_slot = 0;
    }
  }
  return S.next_slot++;
}

void *red_seq_buffer(size_t bytes) {
  RedState &S = rs();
  if (bytes > S.seq_bytes) {
    OP2B_CUDA(cudaStreamSynchronize(rt().stream));
    dev_free(S.seq);
    S.seq = dev_alloc(bytes);
    S.seq_bytes = bytes;
  }
  return S.seq;
}

int red_grid(long long n, int threads) {
  long long want = (n + threads - 1) / threads;
  long long cap = (long long)rt().num_sms * 4;
  if (cap > kMaxRedBlocks) cap = kMaxRedBlocks;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

void red_finish(const std::vector<GblRequest> &reqs) {
  if (reqs.empty()) return;
  if (rt().gbl_deferred) {
    for (auto &r : reqs) pending().push_back(r);
    return;
  }
  deliver(reqs);
  if (pending().empty() && rs().graph_slots == 0) rs().next_slot = 0;
}

void red_finish_after(cudaEvent_t done, const std::vector<GblRequest> &reqs) {
  if (reqs.empty()) return;
  RedState &S = rs();
  OP2B_CUDA(cudaEventSynchronize(done));  // the slots are host memory
  for (auto &r : reqs) {
    const char *p = S.host + (size_t)r.slot * 8;
    if (r.type == GBL_F64) combine<double>(r.host, *(const double *)p, r.acc, r.assign);
    else combine<float>(r.host, *(const float *)p, r.acc, r.assign);
  }
  if (pending().empty() && S.graph_slots == 0) S.next_slot = 0;
}

size_t red_pending_count() { return pending().size(); }

std::vector<GblRequest> red_take_pending_since(size_t mark) {
  std::vector<GblRequest> &p = pending();
  std::vector<GblRequest> out;
  if (mark < p.size()) {
    out.assign(p.begin() + mark, p.end());
    p.resize(mark);
  }
  return out;
}

void red_replace_pending(const std::vector<GblRequest> &reqs) {
  std::vector<GblRequest> &p = pending();
  std::vector<GblRequest> keep;
  for (auto &r : p) {
    bool same = false;
    for (auto &q : reqs) same = same || (q.slot == r.slot);
    if (!same) keep.push_back(r);
  }
  keep.insert(keep.end(), reqs.begin(), reqs.end());
  p.swap(keep);
}

void deliver_deferred() {
  if (pending().empty()) return;
  std::vector<GblRequest> v;
  v.swap(pending());
  deliver(v);
  if (rs().graph_slots == 0) rs().next_slot = 0;
}

void red_reserve_for_graph() { rs().graph_slots = std::max(rs().graph_slots, rs().next_slot); }

}  // namespace op2b

extern "C" int op2b_set_gbl_deferred(int on) {
  op2b::flush_pending();
  op2b::Runtime &R = op2b::rt();
  int old = R.gbl_deferred;
  if (old && !on) op2b::deliver_deferred();
  R.gbl_deferred = on != 0;
  return old;
}
