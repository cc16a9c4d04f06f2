// tile_chain.cuh -- the two phases of the tiled res_calc chain, shared by
// the plain path's k_chain_tiled (airfoil.cu) and the batched form's
// k_grp_chain_tiled (group.cu).
//
// A CTA owns a tile of consecutive cells.  Phase 1 computes, into shared
// memory, the value of every entry of its cells' contribution lists: res_calc's
// flux for an edge, bres_calc's increment for a boundary edge, -0.0 for the
// lists' padding (the identity of addition).  An edge whose cells lie in two
// tiles is computed by both, with the same arithmetic.  Phase 2 folds each
// cell's list from shared memory in list order (op_seq.h's order), applies
// update (airfoil/update.h) and, optionally, save_soln and adt_calc
// (airfoil/save_soln.h, airfoil/adt_calc.h) to the cell.  The per-element
// arithmetic is that of the two-launch chain, term for term, so every field
// is bit-identical to it.
#pragma once

#include "airfoil_math.cuh"

namespace op2b {

// The tile's flux indices (ascending) into shared memory, each in the first
// word of the slot its value will take.  Each thread writes, and later
// reads, only the slots i = threadIdx.x (mod BS).
template <class T, int BS>
__device__ __forceinline__ void tile_stage(const int *__restrict__ tflux, int beg, int cnt, T *fv) {
  int *fidx = reinterpret_cast<int *>(fv);
  constexpr int kSlotInts = 4 * (int)sizeof(T) / (int)sizeof(int);
  for (int i = threadIdx.x; i < cnt; i += BS) fidx[kSlotInts * i] = __ldg(tflux + beg + i);
}

// Phase 1: every staged index's value into its slot, one per thread per
// pass, the next pass's edge map entries fetched while this pass gathers.
// Indices below n_e are edges (pedge, pecell), n_e + b for b < n_b are
// boundary edges (bres(b, r) writes the increment), anything else padding.
template <class T, int BS, class Bres>
__device__ __forceinline__ void tile_fluxes(int cnt, unsigned n_e, unsigned n_b,
                                            const int2 *__restrict__ pedge,
                                            const int2 *__restrict__ pecell,
                                            const T *__restrict__ x, const T *__restrict__ q,
                                            const T *__restrict__ adt, const AirConsts<T> &K,
                                            T *fv, Bres bres) {
  const int *fidx = reinterpret_cast<const int *>(fv);
  constexpr int kSlotInts = 4 * (int)sizeof(T) / (int)sizeof(int);
  int i = threadIdx.x;
  unsigned f = i < cnt ? (unsigned)fidx[kSlotInts * i] : ~0u;
  int2 nn = make_int2(0, 0), cc = make_int2(0, 0);
  if (f < n_e) {
    nn = __ldg(pedge + f);
    cc = __ldg(pecell + f);
  }
  for (; i < cnt; i += BS) {
    const int in = i + BS;
    const unsigned fn = in < cnt ? (unsigned)fidx[kSlotInts * in] : ~0u;
    T r[4];
    if (f < n_e) {
      T p[2], sx[2], q1[4], q2[4];
      ld4(q + 4u * (unsigned)cc.x, q1);
      ld4(q + 4u * (unsigned)cc.y, q2);
      ld2(x + 2u * (unsigned)nn.x, p);
      ld2(x + 2u * (unsigned)nn.y, sx);
      const T d1 = __ldg(adt + (unsigned)cc.x), d2 = __ldg(adt + (unsigned)cc.y);
      if (fn < n_e) {
        nn = __ldg(pedge + fn);
        cc = __ldg(pecell + fn);
      }
      res_flux(p, sx, q1, q2, d1, d2, K.gm1, K.eps, r);
    } else {
      if (f - n_e < n_b) bres((int)(f - n_e), r);
      else r[0] = r[1] = r[2] = r[3] = -T(0);  // the lists' padding value
      if (fn < n_e) {
        nn = __ldg(pedge + fn);
        cc = __ldg(pecell + fn);
      }
    }
    st4(fv + 4 * i, r);
    f = fn;
  }
}

// Phase 2: cells [c0, c1) of the tile, one per thread per pass, the next
// cell's list, nodes and own streams fetched while this one works.  update
// reads qold and adt at the cell and writes the new q to qout (and, SAVE, to
// qsave), res = 0, del^2 to seq (when not null); ADT: adt_calc on the new q
// into adt_out.  res null: res is known to hold +0.0 everywhere (update
// zeroed it and nothing wrote it since), so it is neither read nor
// rewritten; the sums start from the same +0.0.  Returns the thread's sum
// of del^2 in cell order.
template <class T, bool ADT, bool SAVE, int BS>
__device__ __forceinline__ T tile_cells(int c0, int c1, const int *__restrict__ tell, int W,
                                        const int4 *__restrict__ pcell,
                                        const T *__restrict__ xc, const T *qold,
                                        const T *__restrict__ adt, T *__restrict__ qout,
                                        T *__restrict__ res, T *qsave, T *__restrict__ adt_out,
                                        T *seq, const AirConsts<T> &K, const T *fv) {
  T rms = T(0);
  auto fetch = [&](int c, int (&k)[4], int (&nd)[4], T (&r)[4], T (&qo)[4], T &ad) {
    list_head(tell, W, c, k);
    if (ADT) {
      const int4 v = __ldg(pcell + c);
      nd[0] = v.x; nd[1] = v.y; nd[2] = v.z; nd[3] = v.w;
    }
    if (res) ldw4(res + 4 * (size_t)c, r);
    else r[0] = r[1] = r[2] = r[3] = T(0);
    if (SAVE) ldw4(qold + 4 * (size_t)c, qo);  // qsave may be qold itself
    else ld4(qold + 4 * (size_t)c, qo);
    ad = __ldg(adt + c);
  };
  int c = c0 + threadIdx.x;
  int k[4] = {-1, -1, -1, -1}, nd[4] = {0, 0, 0, 0};
  T r[4], qo[4], ad = T(1);
  if (c < c1) fetch(c, k, nd, r, qo, ad);
  for (; c < c1; c += BS) {
    T xs[4][2];
    if (ADT)
#pragma unroll
      for (int j = 0; j < 4; j++) ld2(xc + 2 * (size_t)nd[j], xs[j]);
    const int cn = c + BS;
    int kn[4] = {-1, -1, -1, -1}, ndn[4] = {0, 0, 0, 0};
    T rn[4], qon[4], adn = T(1);
    if (cn < c1) fetch(cn, kn, ndn, rn, qon, adn);
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (k[j] >= 0) {
        T fj[4];
        ldw4(fv + 4 * (k[j] >> 1), fj);
        add_listed(r, k[j], fj);
      }
    for (int j = 4; j < W; j++) {  // lists longer than 4
      const int kk = __ldg(tell + (size_t)c * W + j);
      if (kk < 0) continue;
      T fj[4];
      ldw4(fv + 4 * (kk >> 1), fj);
      add_listed(r, kk, fj);
    }
    // airfoil/update.h:1-12
    const T adti = rcp(ad);
    T qn[4], sq[4];
    for (int d = 0; d < 4; d++) {
      const T del = adti * r[d];
      qn[d] = qo[d] - del;
      sq[d] = del * del;
      rms += sq[d];
    }
    st4(qout + 4 * (size_t)c, qn);
    if (SAVE) st4(qsave + 4 * (size_t)c, qn);  // airfoil/save_soln.h:1-3
    const T z[4] = {T(0), T(0), T(0), T(0)};
    if (res) st4(res + 4 * (size_t)c, z);
    if (seq) st4(seq + 4 * (size_t)c, sq);
    if (ADT) adt_out[c] = adt_calc(xs[0], xs[1], xs[2], xs[3], qn, K);
    if (cn < c1) {
#pragma unroll
      for (int j = 0; j < 4; j++) {
        k[j] = kn[j];
        nd[j] = ndn[j];
        r[j] = rn[j];
        qo[j] = qon[j];
      }
      ad = adn;
    }
  }
  return rms;
}

}  // namespace op2b
