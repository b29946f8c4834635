// spmv_node.cuh -- one node's block row times x, one warp per node (device code
// shared by the one-mesh and the batched Krylov solvers).
//
// The point CSR keeps every node's NEQ rows contiguous over one sorted
// neighbourhood of S nodes: row r of the node holds NEQ*S values starting at
// row_base + r*NEQ*S, column (s, c) at offset s*NEQ + c (s = neighbour slot).
// For NEQ = 4 a lane owns column PAIRS (s, 2h..2h+1): one 16-byte (FP64) or
// 8-byte (FP32) load per row and one for the two x entries, which are
// contiguous because both columns belong to the same neighbour.  NEQ = 3 keeps
// one column per lane.  The NEQ row sums are reduced over the warp with a
// butterfly that halves the number of values per lane in the first two steps
// (6 shuffles instead of 5 per row), in a fixed order, so results are
// deterministic.
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

// Partial row sums of one node's block row: acc[r] += sum over this lane's
// columns of row r.  `row` points at the node's first value, S is the number
// of neighbours (the node itself included), `adj` the node's neighbour list.
template <int NEQ, typename MT, typename VT>
__device__ __forceinline__ void spmv_node_partial(const MT* __restrict__ row, int S, const int32_t* __restrict__ adj,
                                                  const VT* __restrict__ x, int lane, double (&acc)[4]) {
  if constexpr (NEQ == 4) {
    using MP = typename Pair<MT>::type;
    using XP = typename Pair<VT>::type;
    const MP* __restrict__ rp = reinterpret_cast<const MP*>(row);
    const int stride = 2 * S;  // pairs per row
#pragma unroll 1
    for (int p = lane; p < 2 * S; p += 32) {
      const int s = p >> 1;
      const int c0 = (p & 1) * 2;
      const int col = __ldg(adj + s);
      const XP xv = __ldg(reinterpret_cast<const XP*>(x + int64_t(col) * 4 + c0));
      MP v[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) v[r] = __ldcs(rp + (r * stride + p));  // streamed once
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        acc[r] = fma(double(v[r].x), double(xv.x), acc[r]);
        acc[r] = fma(double(v[r].y), double(xv.y), acc[r]);
      }
    }
  } else {
    const int len = NEQ * S;
#pragma unroll 1
    for (int j = lane; j < len; j += 32) {
      const int s = j / NEQ;
      const int c = j - s * NEQ;
      const double xj = double(__ldg(x + int64_t(__ldg(adj + s)) * NEQ + c));
      MT v[NEQ];
#pragma unroll
      for (int r = 0; r < NEQ; ++r) v[r] = __ldcs(row + r * len + j);
#pragma unroll
      for (int r = 0; r < NEQ; ++r) acc[r] = fma(double(v[r]), xj, acc[r]);
    }
  }
}

// y[0..NEQ) of one node = its block row times x (FP64 accumulation), written by
// lanes 0, 8, 16 (, 24).
template <int NEQ, typename MT, typename VT, typename YT>
__device__ __forceinline__ void spmv_node(const MT* __restrict__ row, int S, const int32_t* __restrict__ adj,
                                          const VT* __restrict__ x, int lane, YT* __restrict__ y) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  spmv_node_partial<NEQ, MT, VT>(row, S, adj, x, lane, acc);
  const double sum = warp_sum4(acc, lane);
  const int r = lane >> 3;
  if ((lane & 7) == 0 && r < NEQ) y[r] = YT(sum);
}

// Short block rows (NEQ <= 3: the coupled triangle system, and the velocity
// and pressure systems of the semi-implicit scheme): a warp serves 4 nodes,
// 8 lanes each; lane `sub` of a group owns the neighbours sub, sub + 8, ...:
// their NEQ x entries and the NEQ x NEQ values of each neighbour block.  The
// group's sums are reduced over its 8 lanes in a fixed order; lanes 0..NEQ-1
// of the group write the node's rows.  Every lane of the warp takes part in
// the shuffles (`valid` false: a group past the end).
template <int NEQ, typename MT, typename VT, typename YT>
__device__ __forceinline__ void spmv_node_group(const MT* __restrict__ row, int S, const int32_t* __restrict__ adj,
                                                const VT* __restrict__ x, int sub, bool valid,
                                                YT* __restrict__ y) {
  static_assert(NEQ >= 1 && NEQ <= 3, "8-lane groups serve block rows of 1 to 3 equations");
  constexpr unsigned FULL = 0xffffffffu;
  double acc[NEQ];
#pragma unroll
  for (int r = 0; r < NEQ; ++r) acc[r] = 0.0;
  if (valid) {
    const int len = NEQ * S;
#pragma unroll 1
    for (int s = sub; s < S; s += 8) {
      const int64_t col = __ldg(adj + s);
      double xv[NEQ];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) xv[c] = double(__ldg(x + col * NEQ + c));
#pragma unroll
      for (int r = 0; r < NEQ; ++r)
#pragma unroll
        for (int c = 0; c < NEQ; ++c) acc[r] = fma(double(__ldcs(row + r * len + s * NEQ + c)), xv[c], acc[r]);
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
  if (valid && sub < NEQ) y[sub] = YT(mine);
}

// Triangles of the coupled system (NEQ = 3).
template <typename MT, typename VT, typename YT>
__device__ __forceinline__ void spmv_node3_group(const MT* __restrict__ row, int S, const int32_t* __restrict__ adj,
                                                 const VT* __restrict__ x, int sub, bool valid,
                                                 YT* __restrict__ y) {
  spmv_node_group<3, MT, VT, YT>(row, S, adj, x, sub, valid, y);
}

}  // namespace ufem
