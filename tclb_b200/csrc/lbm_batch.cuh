// Batched iteration of many independent lattices, one launch per iteration
// for all of them.
//
// No counterpart in the reference: TCLB runs one lattice per process. Here
// each case (lattice) has a device descriptor; the cases' nodes are cut into
// uniform tiles listed in a device tile table. By default every tile is one
// thread block (k_iterate_batch_tile), so uneven case sizes balance across
// the SMs through the hardware block scheduler; a persistent grid walking
// the table with a grid stride (k_iterate_batch) is the alternative, slower
// on mixed sizes. The physics is the per-model node update of
// lbm_kernels.cuh, unchanged.
//
// A tile is a bx x by block of nodes of one z plane of one case. With nx a
// multiple of 32 (TCLB's padding) a tile width of 32 leaves no thread idle on
// any case; wider tiles trade that for fewer tiles. The autotuner chooses.
//
// A launch is iteration k (0-based) of a replay of K iterations. A case with
// d = min(remaining, K) iterations to do in this replay runs the last d
// launches, k = K-d .. K-1, so every case's last iteration of a replay is
// launch K-1: that launch alone is the Globals variant, and the plain
// launches carry no Globals code (the register count of the one-lattice
// kernel, not of both paths). Its A/B parity at launch k is
// (counter + k - (K - d)) & 1. The counters advance only in k_batch_advance
// at the end of a replay, so a CUDA graph of K launches + advance can be
// replayed while cases come and go.
#pragma once
#include "lbm_kernels.cuh"

namespace tclb {

constexpr int BATCH_MAX_SET = 16;

struct BatchCase {
  void* buf[2];
  const flag_t* flags;
  const void* zone;  // real_t [zones][NZS]
  double* glob;      // [NG] Globals of the case's last iteration in a replay
  size_t stride;
  int nx, ny, nz;
  int counter;    // iterations done
  int remaining;  // iterations left
  int active;
  double s[BATCH_MAX_SET];
};

struct BatchTile {
  int slot, x0, y0, z;
};

template <class M, class R, class St, bool G>
__global__ void __launch_bounds__(256) k_iterate_batch(const BatchCase* __restrict__ cases,
                                                       const BatchTile* __restrict__ tiles,
                                                       const int* __restrict__ ntiles_p, int k, int K) {
  const int ntiles = *ntiles_p;
  // Chunks of TILE_CHUNK consecutive tiles (usually one case) walked with a
  // grid stride: the case descriptor is read once per chunk and case.
  constexpr int TILE_CHUNK = 4;
  const int nchunks = (ntiles + TILE_CHUNK - 1) / TILE_CHUNK;
  int slot = -1;
  bool skip = true;
  Args<R, M::NSET> a;
  for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int t_end = min(ntiles, (ch + 1) * TILE_CHUNK);
    for (int t = ch * TILE_CHUNK; t < t_end; t++) {
      const BatchTile tile = tiles[t];
      if (tile.slot != slot) {  // uniform across the block
        slot = tile.slot;
        const BatchCase& C = cases[slot];
        const int remaining = C.remaining;
        const int d = remaining < K ? remaining : K;  // this case's iterations in the replay
        const int first = K - d;                      // it runs launches first .. K-1
        skip = !C.active || d <= 0 || k < first;
        const int parity = (C.counter + (k - first)) & 1;
        a.src = C.buf[parity];
        a.dst = C.buf[1 - parity];
        a.stride = C.stride;
        a.flags = C.flags;
        a.nx = C.nx;
        a.ny = C.ny;
        a.nz = C.nz;
        a.zone = static_cast<const R*>(C.zone);
        a.glob = C.glob;
#pragma unroll
        for (int i = 0; i < M::NSET; i++) a.s[i] = (R)C.s[i];
        M::template derived<R>(a.s, a.k);
      }
      if (skip) continue;
      const int x = tile.x0 + threadIdx.x, y = tile.y0 + threadIdx.y, z = tile.z;
      const bool act = x < a.nx && y < a.ny;
      using T = typename St::T;
      const StrideAddr<T> P{static_cast<const T*>(a.src), static_cast<T*>(a.dst), a.stride};
      if constexpr (G) {
        R g[M::NG];
#pragma unroll
        for (int i = 0; i < M::NG; i++) g[i] = 0;
        if (act) node_update<M, R, St, true>(a, P, x, y, z, g);
        reduce_globals<M::NG, M::NSUM, R>(g, a.glob);
        __syncthreads();  // shared scratch of reduce_globals reused by the next tile
      } else {
        if (act) {
          R g[1];
          node_update<M, R, St, false>(a, P, x, y, z, g);
        }
      }
    }
  }
}

// One block per tile (grid = tile-table capacity; blocks past the live tiles
// return at once): blocks are independent, as in the one-lattice kernel.
template <class M, class R, class St, bool G>
__global__ void __launch_bounds__(256, (G || sizeof(R) == 8) ? 1 : M::BATCH_MIN_BLOCKS)
    k_iterate_batch_tile(const BatchCase* __restrict__ cases,
                                                            const BatchTile* __restrict__ tiles,
                                                            const int* __restrict__ ntiles_p, int k, int K) {
  const int t = blockIdx.x;
  if (t >= *ntiles_p) return;
  const BatchTile tile = tiles[t];
  const BatchCase& C = cases[tile.slot];
  const int remaining = C.remaining;
  const int d = remaining < K ? remaining : K;
  const int first = K - d;
  if (!C.active || d <= 0 || k < first) return;
  const int parity = (C.counter + (k - first)) & 1;
  Args<R, M::NSET> a;
  a.src = C.buf[parity];
  a.dst = C.buf[1 - parity];
  a.stride = C.stride;
  a.flags = C.flags;
  a.nx = C.nx;
  a.ny = C.ny;
  a.nz = C.nz;
  a.zone = static_cast<const R*>(C.zone);
  a.glob = C.glob;
#pragma unroll
  for (int i = 0; i < M::NSET; i++) a.s[i] = (R)C.s[i];
  M::template derived<R>(a.s, a.k);
  const int x = tile.x0 + threadIdx.x, y = tile.y0 + threadIdx.y, z = tile.z;
  const bool act = x < a.nx && y < a.ny;
  using T = typename St::T;
  const StrideAddr<T> P{static_cast<const T*>(a.src), static_cast<T*>(a.dst), a.stride};
  if constexpr (G) {
    R g[M::NG];
#pragma unroll
    for (int i = 0; i < M::NG; i++) g[i] = 0;
    if (act) node_update<M, R, St, true>(a, P, x, y, z, g);
    reduce_globals<M::NG, M::NSUM, R>(g, a.glob);
  } else if (act) {
    R g[1];
    node_update<M, R, St, false>(a, P, x, y, z, g);
  }
}

// End of a replay: counters and remaining iterations of every active case.
__global__ void k_batch_advance(BatchCase* cases, int ncases, int K) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncases || !cases[c].active) return;
  const int r = cases[c].remaining;
  const int d = r < K ? r : K;
  cases[c].counter += d;
  cases[c].remaining = r - d;
}

// Clear the Globals of every case at the start of a replay.
template <int NG>
__global__ void k_batch_clear_globals(BatchCase* cases, int ncases) {
  const int c = blockIdx.x;
  if (c >= ncases || !cases[c].active || cases[c].remaining <= 0) return;
  for (int i = threadIdx.x; i < NG; i += blockDim.x) cases[c].glob[i] = 0.0;
}

}  // namespace tclb
