// Device primitives written for this library: an exclusive prefix sum, a stable LSD
// radix sort of (key, value) pairs, and the run boundaries of a sorted key array. The
// Louvain aggregation builds the next level's CSR with them.
//
// Layout shared by all three: a tile is TILE = 256 threads x 8 elements, and warp w of
// a tile owns elements [w * 256, (w + 1) * 256) of it, 32 consecutive elements per step.
// Every load and store of a step is coalesced, and the (warp, step, lane) order of a
// tile's elements is their index order, which is what makes the sort stable.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "sp_internal.cuh"

namespace sp {
namespace prim {

constexpr int T = 256;
constexpr int ITEMS = 8;
constexpr int TILE = T * ITEMS;
constexpr int RADIX = 256;  // 8-bit digits
static_assert(T == RADIX, "one thread per digit in the radix kernels");

template <class V>
__device__ __forceinline__ V warp_inclusive(V x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const V y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Exclusive scan of the TILE values in s (in place), starting from carry; every thread
// gets the tile's total.
template <class V>
__device__ V tile_scan(V* s, V carry) {
  __shared__ V s_warp[T / 32];
  __shared__ V s_total;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  V loc[ITEMS];
  V sum = 0;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    loc[k] = s[t * ITEMS + k];
    sum += loc[k];
  }
  const V inc = warp_inclusive(sum);
  if (lane == 31) s_warp[w] = inc;
  __syncthreads();
  if (t < 32) {
    const V x = t < T / 32 ? s_warp[t] : V(0);
    const V xi = warp_inclusive(x);
    if (t < T / 32) s_warp[t] = xi - x;
    if (t == 31) s_total = xi;
  }
  __syncthreads();
  V run = carry + s_warp[w] + (inc - sum);
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    s[t * ITEMS + k] = run;
    run += loc[k];
  }
  const V total = s_total;
  __syncthreads();
  return total;
}

// part[tile] = sum of the tile's values
template <class V>
__global__ void __launch_bounds__(T) k_tile_sums(const V* __restrict__ in, int64_t n, V* __restrict__ part) {
  __shared__ V s_red[T / 32];
  const int t = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * TILE;
  V sum = 0;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int64_t i = base + k * T + t;
    if (i < n) sum += in[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((t & 31) == 0) s_red[t >> 5] = sum;
  __syncthreads();
  if (t == 0) {
    V tot = 0;
    for (int w = 0; w < T / 32; ++w) tot += s_red[w];
    part[blockIdx.x] = tot;
  }
}

// out[i] = carry[tile] + exclusive scan of the tile (in == out allowed: a tile is read
// whole before it is written)
template <class V>
__global__ void __launch_bounds__(T) k_tile_scan(const V* in, V* out, int64_t n, const V* __restrict__ carry) {
  __shared__ V s[TILE];
  const int t = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * TILE;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int64_t i = base + k * T + t;
    s[k * T + t] = i < n ? in[i] : V(0);
  }
  __syncthreads();
  tile_scan(s, carry ? carry[blockIdx.x] : V(0));
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int64_t i = base + k * T + t;
    if (i < n) out[i] = s[k * T + t];
  }
}

inline int64_t tiles_of(int64_t n) { return (n + TILE - 1) / TILE; }

// Elements of scratch that scan_exclusive needs for n values.
inline int64_t scan_scratch(int64_t n) {
  int64_t need = 0;
  for (int64_t m = tiles_of(n); m > 1; m = tiles_of(m)) need += m;
  return need + 1;
}

// out = exclusive prefix sum of in[0, n); scratch holds scan_scratch(n) values. One
// tile: one launch. More: tile sums, their scan (recursively), and the tiles' scans.
template <class V>
int scan_exclusive(const V* in, V* out, int64_t n, V* scratch, cudaStream_t s) {
  if (n <= 0) return SP_OK;
  const int64_t nt = tiles_of(n);
  if (nt == 1) {
    k_tile_scan<V><<<1, T, 0, s>>>(in, out, n, nullptr);
    SP_CHECK_LAUNCH();
    g_launches += 1;
    return SP_OK;
  }
  V* part = scratch;
  k_tile_sums<V><<<(unsigned)nt, T, 0, s>>>(in, n, part);
  SP_CHECK_LAUNCH();
  SP_TRY(scan_exclusive<V>(part, part, nt, scratch + nt, s));
  k_tile_scan<V><<<(unsigned)nt, T, 0, s>>>(in, out, n, part);
  SP_CHECK_LAUNCH();
  g_launches += 2;
  return SP_OK;
}

// hist[d * ntiles + tile] = elements of the tile whose digit (key >> shift) & 255 is d
template <class K>
__global__ void __launch_bounds__(T) k_radix_hist(const K* __restrict__ keys, int64_t n, int shift,
                                                  int32_t* __restrict__ hist, int ntiles) {
  __shared__ int32_t h[RADIX];
  const int t = threadIdx.x;
  h[t] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * TILE;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int64_t i = base + k * T + t;
    if (i < n) atomicAdd(&h[(int)((keys[i] >> shift) & (RADIX - 1))], 1);
  }
  __syncthreads();
  hist[(int64_t)t * ntiles + blockIdx.x] = h[t];
}

// One stable scatter pass: off = exclusive scan of the digit-major histogram, so an
// element goes to off[d][tile] + (elements of digit d before it in the tile). The rank
// inside a warp step comes from __match_any_sync; warp w's running count per digit
// lives in s_cnt[w][d] and is turned into an offset across the warps of the tile.
template <class K, class V>
__global__ void __launch_bounds__(T) k_radix_scatter(const K* __restrict__ kin, const V* __restrict__ vin,
                                                     K* __restrict__ kout, V* __restrict__ vout, int64_t n,
                                                     int shift, const int32_t* __restrict__ off, int ntiles) {
  __shared__ int32_t s_cnt[T / 32][RADIX];
  __shared__ int32_t s_off[RADIX];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  for (int i = t; i < (T / 32) * RADIX; i += T) (&s_cnt[0][0])[i] = 0;
  s_off[t] = off[(int64_t)t * ntiles + blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * TILE + (int64_t)w * (32 * ITEMS);
  K kk[ITEMS];
  V vv[ITEMS];
  int dd[ITEMS], lp[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int64_t i = base + k * 32 + lane;
    const bool ok = i < n;
    kk[k] = ok ? kin[i] : K(0);
    vv[k] = ok ? vin[i] : V(0);
    const int d = ok ? (int)((kk[k] >> shift) & (RADIX - 1)) : RADIX;  // RADIX: no element
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int before = ok ? s_cnt[w][d] : 0;
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) s_cnt[w][d] = before + __popc(peers);
    __syncwarp();
    dd[k] = d;
    lp[k] = before + __popc(peers & ((1u << lane) - 1u));
  }
  __syncthreads();
  {
    int run = 0;  // thread t: digit t, exclusive over the warps
#pragma unroll
    for (int ww = 0; ww < T / 32; ++ww) {
      const int c = s_cnt[ww][t];
      s_cnt[ww][t] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    if (dd[k] < RADIX) {
      const int64_t p = (int64_t)s_off[dd[k]] + s_cnt[w][dd[k]] + lp[k];
      kout[p] = kk[k];
      vout[p] = vv[k];
    }
  }
}

// Scratch (int32 elements) that radix_sort_pairs needs for n elements.
inline int64_t sort_scratch(int64_t n) {
  const int64_t h = RADIX * tiles_of(n);
  return h + scan_scratch(h);
}

// Stable sort of (keys, vals)[0, n) by key bits [0, end_bit), 8 bits per pass,
// ping-ponging between (k0, v0) (the input) and (k1, v1). *kres / *vres: where the
// sorted pairs are. n < 2^31.
template <class K, class V>
int radix_sort_pairs(K* k0, V* v0, K* k1, V* v1, int64_t n, int end_bit, int32_t* scratch, K** kres, V** vres,
                     cudaStream_t s) {
  *kres = k0;
  *vres = v0;
  if (n <= 1) return SP_OK;
  if (n > INT32_MAX) {
    set_error("radix_sort_pairs: %lld elements", (long long)n);
    return SP_ERR_UNSUPPORTED;
  }
  const int nt = (int)tiles_of(n);
  int32_t* hist = scratch;
  int32_t* rest = scratch + (int64_t)RADIX * nt;
  K* ka = k0;
  V* va = v0;
  K* kb = k1;
  V* vb = v1;
  for (int shift = 0; shift < end_bit; shift += 8) {
    k_radix_hist<K><<<nt, T, 0, s>>>(ka, n, shift, hist, nt);
    SP_CHECK_LAUNCH();
    SP_TRY(scan_exclusive<int32_t>(hist, hist, (int64_t)RADIX * nt, rest, s));
    k_radix_scatter<K, V><<<nt, T, 0, s>>>(ka, va, kb, vb, n, shift, hist, nt);
    SP_CHECK_LAUNCH();
    g_launches += 2;
    K* tk = ka;
    ka = kb;
    kb = tk;
    V* tv = va;
    va = vb;
    vb = tv;
  }
  *kres = ka;
  *vres = va;
  return SP_OK;
}

// head[i] = 1 where a run of equal keys starts (i == 0 or key[i] != key[i - 1]); head[n] = 0
template <class K>
__global__ void k_run_heads(const K* __restrict__ keys, int64_t n, int32_t* __restrict__ head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    head[i] = i < n && (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// start[r] = first index of run r (idx = exclusive scan of head); start[runs] = n
__global__ void k_run_starts(const int32_t* __restrict__ head, const int32_t* __restrict__ idx, int64_t n,
                             int32_t* __restrict__ start) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
    if (i == n)
      start[idx[n]] = (int32_t)n;
    else if (head[i])
      start[idx[i]] = (int32_t)i;
  }
}

}  // namespace prim
}  // namespace sp
