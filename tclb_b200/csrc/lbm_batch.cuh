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
// lbm_kernels.cuh, unchanged. With 16-bit storage the plain launches take
// the two-nodes-per-thread update (k_iterate_batch_pair) and, for cases whose
// rows fit one TMA box, the tile-staged pipeline (k_iterate_batch_tma).
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
// launch K-1: that launch alone is the Globals variant (for the cases that
// compute Globals in this replay: every replay, or with glob_end only the
// finishing one; the others take the plain kernels at K-1 too), and the plain
// launches carry no Globals code (the register count of the one-lattice
// kernel, not of both paths). Its A/B parity at launch k is
// (counter + k - (K - d)) & 1. The counters advance only in k_batch_advance
// at the end of a replay, so a CUDA graph of K launches + advance can be
// replayed while cases come and go.
#pragma once
#include "lbm_kernels.cuh"
#include "lbm_tma.cuh"

namespace tclb {

constexpr int BATCH_MAX_SET = 16;

// Tensor maps of a case for the tile-staged kernel (stored with the case's
// memory): its two snapshots' row maps and its node types.
struct BatchTmaMaps {
  CUtensorMap rows[2], row1[2], flags;
};

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
  int glob_end;               // 1: Globals only in the replay where the case finishes
  int tma_rows;               // rows per staged tile; 0: the case is not staged
  const BatchTmaMaps* maps;   // with tma_rows > 0
  double s[BATCH_MAX_SET];
  double k[4];  // per-case constants derived from s (Model::derived), computed on the host at admission
};

struct BatchTile {
  int slot, x0, y0, z;
  int h;  // rows: the tile is bx x h nodes
};

// A tile of the tile-staged kernel: rows y0 .. y0 + tma_rows - 1 of plane z.
struct BatchTmaTile {
  int slot, z, y0;
};

// Destination planes listed in shared memory (the stores of
// pair_update_store read one pointer each instead of holding Q in registers).
template <class T, int Q>
struct SharedPlanes {
  static constexpr bool per_plane = true;
  T* const* d;
  __device__ __forceinline__ T* dst(int i) const { return d[i]; }
};

// Node-update arguments of a group of cases with the same settings: s[] and
// k[] from the kernel's parameter bank (free operands, as in the
// single-lattice kernels), the zone table from each case.
template <class R, int NSET>
struct GroupArgs {
  typedef R real;
  const R (&s)[NSET];
  const R (&k)[4];
  const R* zone;
};

// Whether case C computes Globals in this replay (of K launches): in every
// replay, or with glob_end only in the one where it finishes.
__device__ __forceinline__ bool case_globals(const BatchCase& C, int K) { return !C.glob_end || C.remaining <= K; }

// Whether case C runs at launch k of a replay of K in a kernel of the
// Globals variant (G) or a plain one, and the A/B parity of that iteration:
// a case with d iterations left runs launches K-d .. K-1. Launch K-1 is its
// last iteration of the replay: the Globals variant takes the cases that
// compute Globals in this replay, the plain kernels the others.
__device__ __forceinline__ bool case_runs(const BatchCase& C, int k, int K, bool G, int& parity) {
  const int remaining = C.remaining;
  const int d = remaining < K ? remaining : K;
  const int first = K - d;
  parity = (C.counter + (k - first)) & 1;
  const bool on = C.active && d > 0 && k >= first;
  return k == K - 1 ? on && G == case_globals(C, K) : on && !G;
}

// The node-update arguments of case C at the given parity (the derived
// constants as the host computed them, so every batch kernel and the staged
// group's parameters use the same values).
template <class M, class R>
__device__ __forceinline__ void case_args(const BatchCase& C, int parity, Args<R, M::NSET>& a) {
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
#pragma unroll
  for (int i = 0; i < 4; i++) a.k[i] = (R)C.k[i];
}

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
        int parity;
        skip = !case_runs(C, k, K, G, parity);
        case_args<M, R>(C, parity, a);
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
template <class M, class R, bool G>
__device__ __forceinline__ bool batch_tile_args(const BatchCase* __restrict__ cases,
                                                const BatchTile* __restrict__ tiles, const int* __restrict__ ntiles_p,
                                                int k, int K, BatchTile& tile, Args<R, M::NSET>& a) {
  const int t = blockIdx.x;
  if (t >= *ntiles_p) return false;
  tile = tiles[t];
  const BatchCase& C = cases[tile.slot];
  int parity;
  if (!case_runs(C, k, K, G, parity)) return false;
  case_args<M, R>(C, parity, a);
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
  if (!batch_tile_args<M, R, G>(cases, tiles, ntiles_p, k, K, tile, a)) return;
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
  if (!batch_tile_args<M, R, false>(cases, tiles, ntiles_p, k, K, tile, a)) return;
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

// 16-bit storage, plain launches, cases whose rows fit one TMA box (see
// tma_rows_for): the tile-staged pipeline of k_iterate_tma over a table of
// tiles of every staged case. For models with the packed collision the
// staged cases are those whose settings equal the group's, ga (so settings
// are parameter-bank operands, as in the single-lattice kernel, and hold no
// registers). Persistent: block b walks tiles b, b + grid, ... The producer
// warp stages each tile's source rows and node types through
// the case's own tensor maps (read from global memory); the consumer warps
// update the tile's node pairs from shared memory. A tile of a case idle at
// this launch is skipped by producer and consumers alike (the same predicate
// on the same descriptor), so both walk the same sequence of stages. A tile
// has R * nx <= 512 nodes (384 when nx = 192): consumer threads past it wait
// and release the stage like the others, so the barrier counts hold. Waits
// are bounded; one that runs out sets *err and the kernel ends.
template <class M, class R, class St>
__global__ void __launch_bounds__(TMA_THREADS, 2)
    k_iterate_batch_tma(const BatchCase* __restrict__ cases, const BatchTmaTile* __restrict__ tiles,
                        const int* __restrict__ ntiles_p, int k, int K, int* err,
                        const __grid_constant__ Args<R, M::NSET> ga) {
  static_assert(M::Q < 32, "one producer lane per population plus one for the node types");
  using P16 = Pack16<St>;
  using T = typename St::T;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);
  constexpr int S = tma_stages<M>();
  static_assert(S <= 8, "128 bytes hold 8 full and 8 empty barriers");
  unsigned long long* empty = full + 8;
  unsigned short* stages = reinterpret_cast<unsigned short*>(smem + 128);
  constexpr unsigned block = TMA_TILE;
  constexpr unsigned stage_elems = (M::Q + 1) * block;
  const int ntiles = *ntiles_p;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int ncons = TMA_CONSUMERS;

  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), ncons);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();  // the only block-wide barrier

  if (warp == ncons) {  // producer
    int n = 0;          // tiles staged so far
    int slot = -1, parity = 0, nx = 0, ny = 0, nz = 0, Rr = 0;
    bool run = false;
    const BatchTmaMaps* mp = nullptr;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const BatchTmaTile tile = tiles[t];
      if (tile.slot != slot) {  // the case's run predicate, parity and shape hold for the launch
        slot = tile.slot;
        const BatchCase& C = cases[slot];
        run = case_runs(C, k, K, false, parity);
        nx = C.nx;
        ny = C.ny;
        nz = C.nz;
        Rr = C.tma_rows;
        mp = C.maps;
        if (run && lane < 3) {  // the three maps this launch uses, into the descriptor cache
          const CUtensorMap* m = lane == 0 ? &mp->rows[parity] : (lane == 1 ? &mp->row1[parity] : &mp->flags);
          asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(m)) : "memory");
        }
      }
      if (!run) continue;
      const int s = n % S;
      const unsigned fb = smem_u32(&full[s]);
      bool ok = true;
      if (lane == 0 && n >= S) ok = mbar_wait(smem_u32(&empty[s]), (unsigned)(n / S - 1) & 1u);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          atomicExch(err, TMA_ERR_TIMEOUT);
          tma_drain(full, S, n, TMA_WAIT_CYCLES);
        }
        return;
      }
      if (lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(fb, (unsigned)(M::Q + 1) * (unsigned)(Rr * tma_pitch(nx)) * 2u);
      }
      __syncwarp();
      tma_fill_at<M>(&mp->rows[parity], &mp->row1[parity], &mp->flags, stages + s * stage_elems, fb, tile.z,
                     tile.y0, nx, ny, nz, Rr, lane);
      n++;
    }
    return;
  }

  // consumers. Models with the packed collision take the settings of the
  // group from ga (the staged cases share them) and the zone table from the
  // case; the others keep the case's arguments in shared memory (one copy per
  // warp, written when the warp's tiles move to another case). Destination
  // planes are listed in shared memory likewise.
  __shared__ Args<R, M::NSET> cargs[TMA_CONSUMERS];
  __shared__ T* cdst[TMA_CONSUMERS][M::Q];
  Args<R, M::NSET>& a = cargs[warp];
  const SharedPlanes<T, M::Q> P{cdst[warp]};
  const R* zone = nullptr;
  int slot = -1, s = 0;
  unsigned phase = 0;
  int nx = 0, ny = 0, r = 0, x = 0;
  bool run = false, act = false;
  // each tile's descriptor is loaded one tile ahead, so its latency overlaps
  // the previous tile's update instead of stalling the warp at every tile
  BatchTmaTile next = (int)blockIdx.x < ntiles ? tiles[blockIdx.x] : BatchTmaTile{0, 0, 0};
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BatchTmaTile tile = next;
    if (t + (int)gridDim.x < ntiles) next = tiles[t + gridDim.x];
    if (tile.slot != slot) {  // the same for every consumer warp
      slot = tile.slot;
      const BatchCase& C = cases[slot];
      int parity;
      run = case_runs(C, k, K, false, parity);
      __syncwarp();
      if constexpr (!M::has_bulk) {
        if (lane == 0) case_args<M, R>(C, parity, a);
      }
      if (lane < M::Q) cdst[warp][lane] = static_cast<T*>(C.buf[1 - parity]) + (size_t)lane * C.stride;
      __syncwarp();
      zone = static_cast<const R*>(C.zone);
      nx = C.nx;
      ny = C.ny;
      const int half = nx >> 1;
      r = tid / half;
      x = 2 * (tid % half);  // a warp may span two rows (nx a multiple of 32)
      act = r < C.tma_rows;
    }
    if (!run) continue;
    const bool ok = mbar_wait(smem_u32(&full[s]), phase);
    if (!__all_sync(0xffffffffu, ok)) {  // the warp leaves together
      if (lane == 0) atomicExch(err, TMA_ERR_TIMEOUT);
      return;
    }
    float2 v[M::Q];
    unsigned fl2 = 0;
    if (act) {
      const unsigned short* mine = stages + s * stage_elems + r * tma_pitch(nx);  // this thread's row, population 0
      // the wrapped neighbours in x, computed here rather than held across tiles
      // (two registers fewer through the collision: no spills)
      const int xm = x == 0 ? nx - 1 : x - 1, xp2 = x + 2 == nx ? 0 : x + 2;
#pragma unroll
      for (int i = 0; i < M::Q; i++) {
        const unsigned short* row = mine + i * block;
        if (M::ex(i) == 0) {
          v[i] = P16::unpack(*reinterpret_cast<const unsigned*>(row + x));
        } else if (M::ex(i) > 0) {  // from x-1
          v[i] = make_float2(P16::lo(row[xm]), P16::lo(row[x]));
        } else {  // from x+1
          v[i] = make_float2(P16::lo(row[x + 1]), P16::lo(row[xp2]));
        }
      }
      fl2 = *reinterpret_cast<const unsigned*>(mine + M::Q * block + x);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&empty[s]));  // this warp is done with the stage
    if (++s == S) {
      s = 0;
      phase ^= 1u;
    }
    if (act) {
      const unsigned node = (unsigned)x + (unsigned)nx * ((unsigned)(tile.y0 + r) + (unsigned)ny * (unsigned)tile.z);
      const flag_t fla = (flag_t)(fl2 & 0xffffu), flb = (flag_t)(fl2 >> 16);
      if constexpr (M::has_bulk) pair_update_store<M, R, St>(v, fla, flb, GroupArgs<R, M::NSET>{ga.s, ga.k, zone}, P, node);
      else pair_update_store<M, R, St>(v, fla, flb, a, P, node);
    }
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

// Clear, at the start of a replay, the Globals of every case that computes
// them in this replay.
template <int NG>
__global__ void k_batch_clear_globals(BatchCase* cases, int ncases, int K) {
  const int c = blockIdx.x;
  if (c >= ncases || !cases[c].active || cases[c].remaining <= 0 || !case_globals(cases[c], K)) return;
  for (int i = threadIdx.x; i < NG; i += blockDim.x) cases[c].glob[i] = 0.0;
}

}  // namespace tclb
