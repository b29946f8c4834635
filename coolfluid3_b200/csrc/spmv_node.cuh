// spmv_node.cuh -- node block rows times x (device code shared by the one-mesh
// and the batched Krylov solvers).
//
// The point CSR keeps every node's NEQ rows contiguous over one sorted
// neighbourhood of S nodes: row r of the node holds NEQ*S values starting at
// row_base + r*NEQ*S, column (s, c) at offset s*NEQ + c (s = neighbour slot).
// NEQ = 4: a warp reduces one node at a time and lane l owns the column PAIRS
// p = l, l + 32, ... (neighbour p / 2, components 2(p % 2) and 2(p % 2) + 1):
// one 16-byte (FP64) or 8-byte (FP32) load per row and one for the two x
// entries, which are contiguous because both columns belong to the same
// neighbour; each pair adds v.x * x.x and then v.y * x.y to the row sums, and
// the NEQ sums are reduced over the warp with a butterfly that halves the
// values per lane in its first two steps (6 shuffles instead of 20).  NEQ <= 3:
// a group of 8 lanes reduces one node, lane `sub` owning the neighbours sub,
// sub + 8, ... (their NEQ x entries and NEQ x NEQ blocks), summed over the
// group by a fixed shuffle tree.  Both walk their nodes with the next node's
// loads in flight.  The order of every sum is fixed, so results are
// deterministic, and FP64 accumulation is used for FP32 operands too.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

namespace ufem {

template <typename T>
struct Pair;
template <>
struct Pair<double> { using type = double2; };
template <>
struct Pair<float> { using type = float2; };

// Sums a[0..3] over the warp.  Afterwards the lanes 8r .. 8r+7 hold the total
// of a[r] (all eight the same value).
__device__ __forceinline__ double warp_sum4(const double (&a)[4], int lane) {
  constexpr unsigned FULL = 0xffffffffu;
  const bool up16 = (lane & 16) != 0;
  const double b0 = (up16 ? a[2] : a[0]) + __shfl_xor_sync(FULL, up16 ? a[0] : a[2], 16);
  const double b1 = (up16 ? a[3] : a[1]) + __shfl_xor_sync(FULL, up16 ? a[1] : a[3], 16);
  const bool up8 = (lane & 8) != 0;
  double c = (up8 ? b1 : b0) + __shfl_xor_sync(FULL, up8 ? b0 : b1, 8);
  c += __shfl_xor_sync(FULL, c, 4);
  c += __shfl_xor_sync(FULL, c, 2);
  c += __shfl_xor_sync(FULL, c, 1);
  return c;
}

// NEQ = 4: the warp's nodes first, first + step, ... < end, with the next
// node's loads in flight: while the warp reduces one node, the neighbour ids
// and values of the next node and the row extent of the node after that are
// already loading, so the chain extent -> values and ids -> x costs one round
// trip a node instead of three.  The prefetched pair is the lane's first; a
// node with more than 16 neighbours loads its further pairs when it is
// reduced.  `first` and `step` are warp-uniform; lanes 0, 8, 16, 24 write the
// node's 4 rows.
template <typename MT, typename VT, typename YT>
__device__ __forceinline__ void spmv4_walk(int64_t first, int64_t end, int64_t step,
                                           const int64_t* __restrict__ start, const int32_t* __restrict__ adj,
                                           const MT* __restrict__ vals, const VT* __restrict__ x,
                                           YT* __restrict__ y, int lane) {
  using MP = typename Pair<MT>::type;
  using XP = typename Pair<VT>::type;
  if (first >= end) return;
  auto extent = [&](int64_t node, int64_t& s0, int& S) {
    if (node < end) {
      s0 = __ldg(start + node);
      S = int(__ldg(start + node + 1) - s0);
    } else {
      s0 = 0;
      S = 0;
    }
  };
  auto load_first = [&](int64_t s0, int S, int& col, MP (&v)[4]) {
    if (lane < 2 * S) {
      col = __ldg(adj + s0 + (lane >> 1));
      const MP* __restrict__ rp = reinterpret_cast<const MP*>(vals + 16 * s0);
#pragma unroll
      for (int r = 0; r < 4; ++r) v[r] = __ldcs(rp + (r * 2 * S + lane));  // streamed once
    }
  };
  int64_t node = first, sA, sB;
  int SA, SB, colA = 0;
  MP vA[4];
  extent(node, sA, SA);
  load_first(sA, SA, colA, vA);
  extent(node + step, sB, SB);
  for (;;) {
    XP xA;
    if (lane < 2 * SA) xA = __ldg(reinterpret_cast<const XP*>(x + int64_t(colA) * 4 + (lane & 1) * 2));
    int colB = 0;
    MP vB[4];
    int64_t sC;
    int SC;
    load_first(sB, SB, colB, vB);  // the next node's first pair (nothing past the end)
    extent(node + 2 * step, sC, SC);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (lane < 2 * SA) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        acc[r] = fma(double(vA[r].x), double(xA.x), acc[r]);
        acc[r] = fma(double(vA[r].y), double(xA.y), acc[r]);
      }
    }
    {  // further pairs of a node with more than 16 neighbours
      const MP* __restrict__ rp = reinterpret_cast<const MP*>(vals + 16 * sA);
      const int stride = 2 * SA;
#pragma unroll 1
      for (int p = lane + 32; p < stride; p += 32) {
        const int col = __ldg(adj + sA + (p >> 1));
        const XP xv = __ldg(reinterpret_cast<const XP*>(x + int64_t(col) * 4 + (p & 1) * 2));
        MP v[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) v[r] = __ldcs(rp + (r * stride + p));
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          acc[r] = fma(double(v[r].x), double(xv.x), acc[r]);
          acc[r] = fma(double(v[r].y), double(xv.y), acc[r]);
        }
      }
    }
    const double sum = warp_sum4(acc, lane);
    if ((lane & 7) == 0) y[node * 4 + (lane >> 3)] = YT(sum);
    node += step;
    if (node >= end) break;
    sA = sB;
    SA = SB;
    colA = colB;
#pragma unroll
    for (int r = 0; r < 4; ++r) vA[r] = vB[r];
    sB = sC;
    SB = SC;
  }
}

// NEQ <= 3: the nodes base + grp for base = n0, n0 + step, ... < n1 (the same
// trip count for every lane of the warp, so every lane takes part in the
// shuffles; `grp` is the lane's group within a step), with the next node's
// extent, first neighbour id and first neighbour block in flight while the
// current node is reduced.  Lanes 0 .. NEQ-1 of a group write its node's rows.
template <int NEQ, typename MT, typename VT, typename YT>
__device__ __forceinline__ void spmv_group_walk(int64_t n0, int64_t n1, int64_t step, int64_t grp, int sub,
                                                const int64_t* __restrict__ start,
                                                const int32_t* __restrict__ adj, const MT* __restrict__ vals,
                                                const VT* __restrict__ x, YT* __restrict__ y) {
  static_assert(NEQ >= 1 && NEQ <= 3, "8-lane groups serve block rows of 1 to 3 equations");
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int NB = NEQ * NEQ;
  auto extent = [&](int64_t node, int64_t& s0, int& S) {
    if (node < n1) {
      s0 = __ldg(start + node);
      S = int(__ldg(start + node + 1) - s0);
    } else {
      s0 = 0;
      S = 0;
    }
  };
  auto load_first = [&](int64_t s0, int S, int64_t& col, MT (&v)[NB]) {
    if (sub < S) {
      col = __ldg(adj + s0 + sub);
      const MT* __restrict__ row = vals + NB * s0;
      const int len = NEQ * S;
#pragma unroll
      for (int r = 0; r < NEQ; ++r)
#pragma unroll
        for (int c = 0; c < NEQ; ++c) v[r * NEQ + c] = __ldcs(row + r * len + sub * NEQ + c);
    }
  };
  int64_t sA, sB, colA = 0;
  int SA, SB;
  MT vA[NB];
  extent(n0 + grp, sA, SA);
  load_first(sA, SA, colA, vA);
  extent(n0 + step + grp, sB, SB);
  for (int64_t base = n0; base < n1; base += step) {
    const int64_t node = base + grp;
    double xv[NEQ];
    if (sub < SA) {
#pragma unroll
      for (int c = 0; c < NEQ; ++c) xv[c] = double(__ldg(x + colA * NEQ + c));
    }
    int64_t colB = 0, sC;
    int SC;
    MT vB[NB];
    load_first(sB, SB, colB, vB);
    extent(base + 2 * step + grp, sC, SC);
    double acc[NEQ];
#pragma unroll
    for (int r = 0; r < NEQ; ++r) acc[r] = 0.0;
    if (sub < SA) {
#pragma unroll
      for (int r = 0; r < NEQ; ++r)
#pragma unroll
        for (int c = 0; c < NEQ; ++c) acc[r] = fma(double(vA[r * NEQ + c]), xv[c], acc[r]);
    }
    {  // further neighbours of a node with more than 8
      const MT* __restrict__ row = vals + NB * sA;
      const int len = NEQ * SA;
#pragma unroll 1
      for (int s = sub + 8; s < SA; s += 8) {
        const int64_t col = __ldg(adj + sA + s);
        double xs[NEQ];
#pragma unroll
        for (int c = 0; c < NEQ; ++c) xs[c] = double(__ldg(x + col * NEQ + c));
#pragma unroll
        for (int r = 0; r < NEQ; ++r)
#pragma unroll
          for (int c = 0; c < NEQ; ++c) acc[r] = fma(double(__ldcs(row + r * len + s * NEQ + c)), xs[c], acc[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < NEQ; ++r) {
      acc[r] += __shfl_xor_sync(FULL, acc[r], 4);
      acc[r] += __shfl_xor_sync(FULL, acc[r], 2);
      acc[r] += __shfl_xor_sync(FULL, acc[r], 1);
    }
    double mine = acc[0];
#pragma unroll
    for (int r = 1; r < NEQ; ++r)
      if (sub == r) mine = acc[r];
    if (node < n1 && sub < NEQ) y[node * NEQ + sub] = YT(mine);
    sA = sB;
    SA = SB;
    colA = colB;
#pragma unroll
    for (int k = 0; k < NB; ++k) vA[k] = vB[k];
    sB = sC;
    SB = SC;
  }
}

}  // namespace ufem
