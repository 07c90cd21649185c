// dvg_device.cuh -- warp / lane-group primitives shared by the kernels.
//
// A "group" is G consecutive lanes of a warp (G in {4, 8, 16, 32}) working on
// one output row.  Every helper takes the group's lane mask; loops whose trip
// count is uniform inside a group keep the group converged, so groups of one
// warp may run different rows with different trip counts.
#pragma once

#include <cstdint>

namespace dvg {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) {
    return kFullMask;
  } else {
    return ((1u << G) - 1u) << (lane_id() & ~(G - 1));
  }
}

template <int G, class T>
__device__ __forceinline__ T group_sum(unsigned m, T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
  return v;
}

template <int G, class T>
__device__ __forceinline__ T group_min(unsigned m, T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    T u = __shfl_xor_sync(m, v, o);
    v = u < v ? u : v;
  }
  return v;
}

template <int G, class T>
__device__ __forceinline__ T group_max(unsigned m, T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    T u = __shfl_xor_sync(m, v, o);
    v = u > v ? u : v;
  }
  return v;
}

// Inclusive prefix sum / max over the lanes of a group (lane order).
template <int G, class T>
__device__ __forceinline__ T group_incl_sum(unsigned m, T v, int lg) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    T u = __shfl_up_sync(m, v, o, G);
    if (lg >= o) v += u;
  }
  return v;
}

template <int G, class T>
__device__ __forceinline__ T group_incl_max(unsigned m, T v, int lg) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    T u = __shfl_up_sync(m, v, o, G);
    if (lg >= o && u > v) v = u;
  }
  return v;
}

// Value of `v` held by group lane `src`.
template <int G, class T>
__device__ __forceinline__ T group_bcast(unsigned m, T v, int src) {
  return __shfl_sync(m, v, src, G);
}

// 8-byte load of one [start, end] range (entries of a row start at an even
// index, so a range is 8-byte aligned in an 8-byte aligned array).
__device__ __forceinline__ uint2 load_range(const uint32_t* __restrict__ entries, uint64_t range_idx) {
  return __ldg(reinterpret_cast<const uint2*>(entries) + range_idx);
}

}  // namespace dvg
