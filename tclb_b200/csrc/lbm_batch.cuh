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
// any case; wider tiles trade that for fewer tiles. A thread block has at
// most 256 threads (bx x min(by, 256 / bx)) and walks the tile's rows, so a
// taller tile spreads the block's descriptor reads over more nodes. The
// autotuner chooses the shape; the tile table lowers the height when the live
// cases would give too few tiles to fill the GPU.
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
  int h;  // rows: the tile is bx x h nodes
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
      const int x = tile.x0 + threadIdx.x, z = tile.z;
      const int y_end = min(tile.y0 + tile.h, a.ny);
      using T = typename St::T;
      const StrideAddr<T> P{static_cast<const T*>(a.src), static_cast<T*>(a.dst), a.stride};
      if constexpr (G) {
        R g[M::NG];
#pragma unroll
        for (int i = 0; i < M::NG; i++) g[i] = 0;
        if (x < a.nx)
          for (int y = tile.y0 + threadIdx.y; y < y_end; y += blockDim.y) node_update<M, R, St, true>(a, P, x, y, z, g);
        reduce_globals<M::NG, M::NSUM, R>(g, a.glob);
        __syncthreads();  // shared scratch of reduce_globals reused by the next tile
      } else if (x < a.nx) {
        R g[1];
        for (int y = tile.y0 + threadIdx.y; y < y_end; y += blockDim.y) node_update<M, R, St, false>(a, P, x, y, z, g);
      }
    }
  }
}

// The arguments of tile t at launch k of a replay of K; false if the block
// has nothing to do (past the live tiles, or the case idle at this launch).
template <class M, class R>
__device__ __forceinline__ bool batch_tile_args(const BatchCase* __restrict__ cases,
                                                const BatchTile* __restrict__ tiles, const int* __restrict__ ntiles_p,
                                                int k, int K, BatchTile& tile, Args<R, M::NSET>& a) {
  const int t = blockIdx.x;
  if (t >= *ntiles_p) return false;
  tile = tiles[t];
  const BatchCase& C = cases[tile.slot];
  const int remaining = C.remaining;
  const int d = remaining < K ? remaining : K;
  const int first = K - d;
  if (!C.active || d <= 0 || k < first) return false;
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
  return true;
}

// One block per tile (grid = live tiles): blocks are independent, as in the
// one-lattice kernel. A block of bx x by threads walks the tile's h rows with
// stride by, so its descriptor reads are spread over h / by nodes per thread.
template <class M, class R, class St, bool G>
__global__ void __launch_bounds__(256, (G || sizeof(R) == 8) ? 1 : M::BATCH_MIN_BLOCKS)
    k_iterate_batch_tile(const BatchCase* __restrict__ cases, const BatchTile* __restrict__ tiles,
                         const int* __restrict__ ntiles_p, int k, int K) {
  BatchTile tile;
  Args<R, M::NSET> a;
  if (!batch_tile_args<M, R>(cases, tiles, ntiles_p, k, K, tile, a)) return;
  const int x = tile.x0 + threadIdx.x, z = tile.z;
  const int y_end = min(tile.y0 + tile.h, a.ny);
  using T = typename St::T;
  const StrideAddr<T> P{static_cast<const T*>(a.src), static_cast<T*>(a.dst), a.stride};
  if constexpr (G) {
    R g[M::NG];
#pragma unroll
    for (int i = 0; i < M::NG; i++) g[i] = 0;
    if (x < a.nx)
      for (int y = tile.y0 + threadIdx.y; y < y_end; y += blockDim.y) node_update<M, R, St, true>(a, P, x, y, z, g);
    reduce_globals<M::NG, M::NSUM, R>(g, a.glob);
  } else if (x < a.nx) {
    R g[1];
    for (int y = tile.y0 + threadIdx.y; y < y_end; y += blockDim.y) node_update<M, R, St, false>(a, P, x, y, z, g);
  }
}

// 16-bit storage, plain launches: two neighbouring nodes per thread with
// 32-bit accesses, the update of the one-lattice pair kernel. A tile of
// bx x h nodes (bx a multiple of 64) runs as a block of bx / 2 x by threads
// walking the rows with stride by; each warp covers 64 consecutive x of one
// row. In the last tile of a row whose width is not a
// multiple of 64 the lanes past the row only load (node_update_pair's
// PARTIAL form). A case with odd nx has no node pairs: its tiles take the
// one-node update, two nodes per thread.
template <class M, class R, class St>
__global__ void __launch_bounds__(M::PAIR_THREADS, M::PAIR_MIN_BLOCKS)
    k_iterate_batch_pair(const BatchCase* __restrict__ cases, const BatchTile* __restrict__ tiles,
                         const int* __restrict__ ntiles_p, int k, int K) {
  BatchTile tile;
  Args<R, M::NSET> a;
  if (!batch_tile_args<M, R>(cases, tiles, ntiles_p, k, K, tile, a)) return;
  using T = typename St::T;
  const StrideAddr<T> P{static_cast<const T*>(a.src), static_cast<T*>(a.dst), a.stride};
  const int z = tile.z;
  const int y_end = min(tile.y0 + tile.h, a.ny);  // y is uniform per warp: a warp lies in one row
  if (a.nx & 1) {
    R g[1];
    for (int y = tile.y0 + threadIdx.y; y < y_end; y += blockDim.y)
      for (int x = tile.x0 + threadIdx.x; x < tile.x0 + 2 * (int)blockDim.x && x < a.nx; x += blockDim.x)
        node_update<M, R, St, false>(a, P, x, y, z, g);
    return;
  }
  const int x = tile.x0 + 2 * threadIdx.x;
  for (int y = tile.y0 + threadIdx.y; y < y_end; y += blockDim.y)
    node_update_pair<M, R, St, StrideAddr<T>, true>(a, P, x, y, z, threadIdx.x & 31);
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
