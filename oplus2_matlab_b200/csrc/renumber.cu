// renumber.cu -- optional renumbering of every set for locality of the
// indirect gathers (op2b_set_renumber).
//
// A mesh whose numbering is scrambled turns each gather into a random
// access.  When renumbering is on, the first loop call orders every set:
//  - the anchor set is the one most maps point to (ties: the larger);
//    elements that share a row of a map of dim >= 2 onto it are neighbours,
//    and a breadth-first walk (Cuthill-McKee, from a least-connected element
//    of each connected component) gives its order;
//  - every set with a map onto an ordered set follows: its elements sorted
//    by the smallest new index they point to (ties by old index);
//  - a set only pointed to by an ordered set takes the order in which the
//    ordered set's rows first reach it;
//  - anything left keeps its numbering.
// Each dataset is then stored permuted on the device (element i of the new
// order is element P[i] of the app's), each map's device copy has its rows
// in the new order of its from-set and its values in the new numbering of
// its to-set, and op_fetch_data puts the app's order back.
//
// Results do not change: per-element arithmetic is the same, and the
// owner-computes plans order each target's contributions by the APP's
// element numbers (get_gather_plan sorts by original keys), which is still
// op_seq.h's order.  Global sums in TREE mode are summed in another order
// (as with any launch shape); plans returned by op_plan_get describe the
// renumbered sets.

#include <limits.h>

#include <algorithm>
#include <queue>
#include <vector>

#include "internal.h"
#include "plan.h"

namespace op2b {

namespace {

struct SetPerm {
  std::vector<int> P, Q;  // new -> old, old -> new
  int *d_P = nullptr, *d_Q = nullptr;
};

std::vector<SetPerm> g_perm;  // by set index; empty P: not permuted
bool g_enabled = false, g_applied = false, g_computed = false;

bool permuted(int set_index) {
  return set_index < (int)g_perm.size() && !g_perm[set_index].P.empty();
}

// Cuthill-McKee order of the anchor set's neighbour graph
std::vector<int> anchor_order(op_set s) {
  const int n = s->size;
  std::vector<int> deg(n, 0);
  std::vector<op_map> onto;
  for (int k = 0; k < OP_map_index; k++) {
    op_map m = OP_map_list[k];
    if (m->to == s && m->dim >= 2) onto.push_back(m);
  }
  // neighbour lists: every pair in a row
  for (op_map m : onto)
    for (int r = 0; r < m->from->size; r++)
      for (int a = 0; a < m->dim; a++) deg[m->map[(size_t)r * m->dim + a]] += m->dim - 1;
  std::vector<long long> off(n + 1, 0);
  for (int i = 0; i < n; i++) off[i + 1] = off[i] + deg[i];
  std::vector<int> adj(off[n]);
  std::vector<long long> cur(off.begin(), off.end() - 1);
  for (op_map m : onto)
    for (int r = 0; r < m->from->size; r++) {
      const int *row = m->map + (size_t)r * m->dim;
      for (int a = 0; a < m->dim; a++)
        for (int b = 0; b < m->dim; b++)
          if (a != b) adj[cur[row[a]]++] = row[b];
    }
  std::vector<int> order;
  order.reserve(n);
  std::vector<char> seen(n, 0);
  // start each component at a least-connected element, found in one pass
  std::vector<int> by_deg(n);
  for (int i = 0; i < n; i++) by_deg[i] = i;
  std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
  for (int start : by_deg) {
    if (seen[start]) continue;
    std::queue<int> q;
    q.push(start);
    seen[start] = 1;
    while (!q.empty()) {
      const int v = q.front();
      q.pop();
      order.push_back(v);
      for (long long j = off[v]; j < off[v + 1]; j++) {
        const int w = adj[j];
        if (!seen[w]) {
          seen[w] = 1;
          q.push(w);
        }
      }
    }
  }
  return order;
}

void set_perm(op_set s, std::vector<int> P) {
  if ((int)g_perm.size() <= s->index) g_perm.resize(s->index + 1);
  SetPerm &sp = g_perm[s->index];
  sp.Q.assign(P.size(), 0);
  for (size_t i = 0; i < P.size(); i++) sp.Q[P[i]] = (int)i;
  sp.P = std::move(P);
}

void compute_orders() {
  g_perm.clear();
  g_perm.resize(OP_set_index);
  if (OP_set_index == 0) return;
  // anchor: most maps onto it, then the larger
  op_set anchor = nullptr;
  int best = -1;
  for (int k = 0; k < OP_set_index; k++) {
    op_set s = OP_set_list[k];
    int score = 0;
    for (int j = 0; j < OP_map_index; j++)
      if (OP_map_list[j]->to == s && OP_map_list[j]->dim >= 2) score++;
    if (score > best || (score == best && anchor && s->size > anchor->size)) {
      best = score;
      anchor = s;
    }
  }
  if (best <= 0) return;  // no map with shared rows: nothing to gain
  set_perm(anchor, anchor_order(anchor));
  bool progress = true;
  while (progress) {
    progress = false;
    for (int k = 0; k < OP_set_index; k++) {
      op_set s = OP_set_list[k];
      if (permuted(s->index) || s->size == 0) continue;
      // a map from s onto an ordered set
      op_map via = nullptr;
      for (int j = 0; j < OP_map_index && !via; j++) {
        op_map m = OP_map_list[j];
        if (m->from == s && permuted(m->to->index)) via = m;
      }
      if (via) {
        const std::vector<int> &Qt = g_perm[via->to->index].Q;
        std::vector<int> key(s->size);
        for (int e = 0; e < s->size; e++) {
          int mn = INT_MAX;
          for (int a = 0; a < via->dim; a++)
            mn = std::min(mn, Qt[via->map[(size_t)e * via->dim + a]]);
          key[e] = mn;
        }
        std::vector<int> P(s->size);
        for (int e = 0; e < s->size; e++) P[e] = e;
        std::stable_sort(P.begin(), P.end(), [&](int a, int b) { return key[a] < key[b]; });
        set_perm(s, std::move(P));
        progress = true;
        continue;
      }
      // a map from an ordered set onto s
      for (int j = 0; j < OP_map_index; j++) {
        op_map m = OP_map_list[j];
        if (m->to != s || !permuted(m->from->index)) continue;
        const std::vector<int> &Pf = g_perm[m->from->index].P;
        std::vector<char> seen(s->size, 0);
        std::vector<int> P;
        P.reserve(s->size);
        for (int r : Pf)
          for (int a = 0; a < m->dim; a++) {
            const int v = m->map[(size_t)r * m->dim + a];
            if (!seen[v]) {
              seen[v] = 1;
              P.push_back(v);
            }
          }
        for (int v = 0; v < s->size; v++)
          if (!seen[v]) P.push_back(v);
        set_perm(s, std::move(P));
        progress = true;
        break;
      }
    }
  }
  g_computed = true;
}

// out[i] = in[P[i]] (forward) or out[P[i]] = in[i] (back), w words per element
__global__ void k_permute(const unsigned *__restrict__ in, unsigned *__restrict__ out,
                          const int *__restrict__ P, long long n, int w, int back) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * w;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / w;
    const int c = (int)(t % w);
    const long long p = P[i];
    if (back) out[p * w + c] = in[i * w + c];
    else out[i * w + c] = in[p * w + c];
  }
}

__global__ void k_permute_bytes(const unsigned char *__restrict__ in, unsigned char *__restrict__ out,
                                const int *__restrict__ P, long long n, int w, int back) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * w;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / w;
    const int c = (int)(t % w);
    const long long p = P[i];
    if (back) out[p * w + c] = in[i * w + c];
    else out[i * w + c] = in[p * w + c];
  }
}

void permute_launch(const void *in, void *out, const int *dP, long long n, int size, int back) {
  cudaStream_t s = rt().stream;
  const int grid = rt().num_sms * 8;
  if (size % 4 == 0)
    k_permute<<<grid, 256, 0, s>>>((const unsigned *)in, (unsigned *)out, dP, n, size / 4, back);
  else
    k_permute_bytes<<<grid, 256, 0, s>>>((const unsigned char *)in, (unsigned char *)out, dP, n,
                                         size, back);
}

}  // namespace

bool renumber_enabled() { return g_enabled; }

// the set's device permutation (new -> old / old -> new), or nullptr
const int *perm_new2old_dev(op_set s) {
  return s && permuted(s->index) && g_applied ? g_perm[s->index].d_P : nullptr;
}
const int *perm_old2new_dev(op_set s) {
  return s && permuted(s->index) && g_applied ? g_perm[s->index].d_Q : nullptr;
}

// store a dataset of a renumbered set in the new order (in place)
void permute_dat_in_place(op_dat d) {
  if (!d || !d->data_d || !perm_new2old_dev(d->set)) return;
  const size_t bytes = (size_t)d->size * d->set->size;
  void *tmp = dev_alloc(bytes);
  if (!tmp) return;
  permute_launch(d->data_d, tmp, perm_new2old_dev(d->set), d->set->size, d->size, 0);
  OP2B_CUDA(cudaMemcpyAsync(d->data_d, tmp, bytes, cudaMemcpyDeviceToDevice, rt().stream));
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  dev_free(tmp);
}

// device data of `d` in the app's order into host memory
bool fetch_unpermuted(op_dat d, void *host) {
  if (!d || !perm_new2old_dev(d->set)) return false;
  const size_t bytes = (size_t)d->size * d->set->size;
  void *tmp = dev_alloc(bytes);
  if (!tmp) return true;
  permute_launch(d->data_d, tmp, perm_new2old_dev(d->set), d->set->size, d->size, 1);
  OP2B_CUDA(cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, rt().stream));
  OP2B_CUDA(cudaStreamSynchronize(rt().stream));
  dev_free(tmp);
  return true;
}

// host copy of a map in the renumbered order, or empty when unchanged
std::vector<int> renumbered_map(op_map m) {
  std::vector<int> out;
  if (!g_applied) return out;
  const bool pf = permuted(m->from->index), pt = permuted(m->to->index);
  if (!pf && !pt) return out;
  const int n = m->from->size, dim = m->dim;
  out.resize((size_t)n * dim);
  for (int i = 0; i < n; i++) {
    const int src = pf ? g_perm[m->from->index].P[i] : i;
    for (int a = 0; a < dim; a++) {
      const int v = m->map[(size_t)src * dim + a];
      out[(size_t)i * dim + a] = pt ? g_perm[m->to->index].Q[v] : v;
    }
  }
  return out;
}

void release_plans_and_maps();  // device.cu

// called by the first loop call: order the sets, move the data
void renumber_apply() {
  if (!g_enabled || g_applied) return;
  compute_orders();  // from the sets and maps declared by now
  for (int k = 0; k < (int)g_perm.size(); k++) {
    SetPerm &sp = g_perm[k];
    if (sp.P.empty()) continue;
    sp.d_P = (int *)dev_alloc(sizeof(int) * sp.P.size());
    sp.d_Q = (int *)dev_alloc(sizeof(int) * sp.Q.size());
    if (!sp.d_P || !sp.d_Q) return;
    OP2B_CUDA(cudaMemcpy(sp.d_P, sp.P.data(), sizeof(int) * sp.P.size(), cudaMemcpyHostToDevice));
    OP2B_CUDA(cudaMemcpy(sp.d_Q, sp.Q.data(), sizeof(int) * sp.Q.size(), cudaMemcpyHostToDevice));
  }
  g_applied = true;
  release_plans_and_maps();  // device copies of maps and plans follow the new order
  for (int k = 0; k < OP_dat_index; k++) permute_dat_in_place(OP_dat_list[k]);
}

void renumber_reset() {
  for (auto &sp : g_perm) {
    dev_free(sp.d_P);
    dev_free(sp.d_Q);
  }
  g_perm.clear();
  g_applied = g_computed = false;
  g_enabled = false;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

int op2b_set_renumber(int on) {
  if (g_applied && !on) {
    fail(-1, "op2b error -- renumbering cannot be turned off after the first loop\n");
    return -1;
  }
  g_enabled = on != 0;
  return 0;
}

int op2b_renumber_order(op_set set, int *new2old) {
  if (!set || !new2old) return -1;
  if (!g_applied) compute_orders();
  if (permuted(set->index)) {
    std::copy(g_perm[set->index].P.begin(), g_perm[set->index].P.end(), new2old);
    return 1;
  }
  for (int i = 0; i < set->size; i++) new2old[i] = i;
  return 0;
}

}  // extern "C"
