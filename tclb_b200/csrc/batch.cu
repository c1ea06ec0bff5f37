// Batched lattices: many independent cases of one model advanced by one
// launch per iteration, K iterations per CUDA-graph replay. New API (no
// counterpart in the reference, which runs one lattice per process).
//
// Memory: each case is one allocation from a stream-ordered CUDA memory pool
// owned by the batch (two snapshots, node types, zonal settings, Globals and,
// for a case the tile-staged kernel can take, its tensor maps), so
// admitting and retiring cases never synchronises the device. A byte budget
// bounds the sum of case footprints; admission beyond it is refused.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/tclb_b200.h"
#include "lbm_batch.cuh"

using namespace tclb;

namespace {

thread_local std::string g_batch_err;

int bfail(int code, const std::string& msg) {
  g_batch_err = msg;
  return code;
}

#define BCK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return bfail(TCLB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Kernel forms of the iteration launches.
enum BatchForm { FORM_PERSISTENT = 0, FORM_TILE = 1, FORM_PAIR = 2 };

// The device tables a replay's launches read.
struct LaunchTables {
  const BatchCase* cases;
  const BatchTile* tiles;      // tiles of the cases not staged, then those of the staged cases
  const int* ntiles;           // [0] tiles of the cases not staged, [1] all tiles
  const BatchTmaTile* ttiles;  // tiles of the tile-staged kernel
  const int* nttiles;
  int* err;                    // set by a staging wait that ran out
};

struct BatchImpl {
  // Launch k of K. Plain launches: the tile-staged kernel over the staged
  // cases when tma_grid > 0, then the plain form over the other cases' tiles
  // (grid gp); FORM_PAIR takes the pair kernel (bx / 2 threads per row). The
  // Globals launch (k = K-1): the one-tile kernel over every case's tiles
  // (grid ga, bx threads per row).
  // group: the settings shared by the staged cases (models with the packed
  // collision; see tclb_batch::group)
  // plain_last: launch K-1 also runs the plain kernels, for the cases that
  // compute no Globals in this replay (TCLB_BATCH_GLOBALS_AT_END)
  void (*iterate)(const LaunchTables&, int k, int K, dim3 gp, dim3 ga, int tma_grid, const double* group, int bx,
                  int by, int form, bool plain_last, cudaStream_t);
  // resident blocks of the tile-staged kernel on the device (it also sets the
  // kernel's shared-memory limit); 0 without one
  int (*tma_grid)(int sms);
  // the derived constants k of a case from its settings (host, in real_t)
  void (*derive)(BatchCase&);
  void (*clear)(BatchCase*, int n, int K, cudaStream_t);
  void (*init)(const BatchCase&, const void* dst, cudaStream_t, int bx, int by);
  void (*quantity)(const BatchCase&, int parity, int q, int vec, double scale, void* out, cudaStream_t);
  int (*blocks_per_sm)(int threads);
  const void* (*tile_kernel)(int which);  // 0 one-tile plain, 1 one-tile Globals, 2 pair
  int pair_threads;                        // block-size limit of the pair kernel; 0: no pair kernel
  bool group_staging;                      // staged cases must share their settings (packed collision)
  // smallest staged tile (nodes) of a case; cases with smaller tiles take the
  // register kernels (0: any tile)
  int min_staged_nodes;
  size_t real_size;
  int Q, NG, NSET, NZS, zone_shift;
};

// Thread rows of a block for tiles bx x by nodes with at most max_threads
// threads: the block walks the remaining rows.
int block_rows(int bx, int by, int max_threads) { return std::max(1, std::min(by, max_threads / bx)); }

template <class M, class R>
Args<R, M::NSET> args_of(const BatchCase& C, const void* src, void* dst) {
  Args<R, M::NSET> a;
  a.src = src;
  a.dst = dst;
  a.stride = C.stride;
  a.flags = C.flags;
  a.nx = C.nx;
  a.ny = C.ny;
  a.nz = C.nz;
  a.zone = static_cast<const R*>(C.zone);
  a.glob = C.glob;
  for (int i = 0; i < M::NSET; i++) a.s[i] = (R)C.s[i];
  M::template derived<R>(a.s, a.k);
  return a;
}

template <class M, class R, class St>
struct BL {
  // launch K-1 of a replay is every case's last iteration: the Globals variant
  static constexpr bool pairs = sizeof(typename St::T) == 2;  // 16-bit storage
  static size_t tma_smem() { return tma_smem_bytes<M>(); }
  static void iterate(const LaunchTables& L, int k, int K, dim3 gp, dim3 ga, int tma_grid, const double* group,
                      int bx, int by, int form, bool plain_last, cudaStream_t s) {
    const dim3 b(bx, block_rows(bx, by, 256));
    const BatchCase* c = L.cases;
    const BatchTile* t = L.tiles;
    if (k == K - 1) {  // every case's last iteration of the replay: the Globals variant, all tiles
      if (form == FORM_PERSISTENT) k_iterate_batch<M, R, St, true><<<gp, b, 0, s>>>(c, t, L.ntiles + 1, k, K);
      else k_iterate_batch_tile<M, R, St, true><<<ga, b, 0, s>>>(c, t, L.ntiles + 1, k, K);
      if (!plain_last) return;
    }
    if constexpr (pairs) {
      if (tma_grid > 0) {
        BatchCase G;  // the group's settings and derived constants
        std::memset(&G, 0, sizeof(G));
        if (group)
          for (int i = 0; i < M::NSET; i++) G.s[i] = group[i];
        const Args<R, M::NSET> gargs = args_of<M, R>(G, nullptr, nullptr);
        k_iterate_batch_tma<M, R, St>
            <<<tma_grid, TMA_THREADS, tma_smem(), s>>>(c, L.ttiles, L.nttiles, k, K, L.err, gargs);
      }
      if (form == FORM_PAIR) {
        const dim3 bp(bx / 2, block_rows(bx / 2, by, M::PAIR_THREADS));
        k_iterate_batch_pair<M, R, St><<<gp, bp, 0, s>>>(c, t, L.ntiles, k, K);
        return;
      }
    }
    if (form == FORM_PERSISTENT) k_iterate_batch<M, R, St, false><<<gp, b, 0, s>>>(c, t, L.ntiles, k, K);
    else k_iterate_batch_tile<M, R, St, false><<<gp, b, 0, s>>>(c, t, L.ntiles, k, K);
  }
  static void derive(BatchCase& C) {
    const Args<R, M::NSET> a = args_of<M, R>(C, nullptr, nullptr);
    for (int i = 0; i < 4; i++) C.k[i] = (double)a.k[i];
  }
  static int tma_grid(int sms) {
    if constexpr (pairs) {
      const void* f = reinterpret_cast<const void*>(k_iterate_batch_tma<M, R, St>);
      int n = 0;
      if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem()) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, TMA_THREADS, tma_smem()) != cudaSuccess) {
        cudaGetLastError();
        return 0;
      }
      return n * sms;
    }
    return 0;
  }
  static const void* tile_kernel(int which) {
    if constexpr (pairs) {
      if (which == 2) return reinterpret_cast<const void*>(k_iterate_batch_pair<M, R, St>);
    }
    if (which == 2) return nullptr;
    return which ? reinterpret_cast<const void*>(k_iterate_batch_tile<M, R, St, true>)
                 : reinterpret_cast<const void*>(k_iterate_batch_tile<M, R, St, false>);
  }
  // resident blocks per SM of the plain kernel at this block size
  static int blocks_per_sm(int threads) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_iterate_batch<M, R, St, false>, threads, 0) !=
        cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return n;
  }
  static void clear(BatchCase* c, int n, int K, cudaStream_t s) {
    if (n > 0) k_batch_clear_globals<M::NG><<<n, 32, 0, s>>>(c, n, K);
  }
  static void init(const BatchCase& C, const void* dst, cudaStream_t s, int bx, int by) {
    auto a = args_of<M, R>(C, nullptr, const_cast<void*>(dst));
    dim3 grd((C.nx + bx - 1) / bx, (C.ny + by - 1) / by, C.nz);
    k_init<M, R, St><<<grd, dim3(bx, by), 0, s>>>(a);
  }
  static void quantity(const BatchCase& C, int parity, int q, int vec, double scale, void* out, cudaStream_t s) {
    auto a = args_of<M, R>(C, C.buf[parity], nullptr);
    dim3 grd((C.nx + 31) / 32, (C.ny + 3) / 4, C.nz);
    k_quantity<M, R, St><<<grd, dim3(32, 4), 0, s>>>(a, q, vec, 0, 0, 0, C.nx, C.ny, C.nz, (R)scale,
                                                      static_cast<R*>(out));
  }
  // d3q19's register pair kernel (identity-rate lanes) measured faster than
  // staged tiles that leave more than an eighth of the consumer threads idle
  // (B200, porous boxes in batches: edge 160, 320-node tiles: 43.4k against
  // 38.9k MLUPS; edge 192, 384-node tiles: 49.7k against 42.0k)
  static constexpr int min_staged_nodes() { return M::identity_lanes ? 448 : 0; }
  static const BatchImpl* get() {
    static const BatchImpl impl = {iterate,
                                   tma_grid,
                                   derive,
                                   clear,
                                   init,
                                   quantity,
                                   blocks_per_sm,
                                   tile_kernel,
                                   pairs ? M::PAIR_THREADS : 0,
                                   M::has_bulk,
                                   min_staged_nodes(),
                                   sizeof(R),
                                   M::Q,
                                   M::NG,
                                   M::NSET,
                                   M::NZS,
                                   M::ZONE_SHIFT};
    return &impl;
  }
};

template <class M>
const BatchImpl* bimpl_model(int precision, int storage) {
  if (precision == TCLB_FP64) return storage == TCLB_STORAGE_SAME ? BL<M, double, StoreF64>::get() : nullptr;
  switch (storage) {
    case TCLB_STORAGE_SAME: return BL<M, float, StoreF32>::get();
    case TCLB_STORAGE_FP16: return BL<M, float, StoreF16<false>>::get();
    case TCLB_STORAGE_FP16_SHIFT: return BL<M, float, StoreF16<true>>::get();
    case TCLB_STORAGE_BF16: return BL<M, float, StoreBF16<false>>::get();
    case TCLB_STORAGE_BF16_SHIFT: return BL<M, float, StoreBF16<true>>::get();
  }
  return nullptr;
}

const BatchImpl* bimpl(int model, int precision, int storage) {
  switch (model) {
    case MODEL_D2Q9: return bimpl_model<D2Q9>(precision, storage);
    case MODEL_D3Q19: return bimpl_model<D3Q19>(precision, storage);
    case MODEL_D3Q27C: return bimpl_model<D3Q27C>(precision, storage);
  }
  return nullptr;
}

size_t elem_size(int precision, int storage) {
  return precision == TCLB_FP64 ? 8 : (storage == TCLB_STORAGE_SAME ? 4 : 2);
}

struct CaseLayout {
  size_t stride, buf, flags, zone, glob, maps, total;
};

// Rows per staged tile of a case (tma_rows_for), or 0 where the case takes
// the register kernels: its rows do not fit a box, or its tiles are smaller
// than the model's min_staged_nodes.
int staged_rows(const BatchImpl* I, size_t elem, int nx, int ny) {
  const int R = tma_rows_for(elem, nx, ny);
  return R * nx >= I->min_staged_nodes ? R : 0;
}

// One allocation per case: two snapshots, node types, zone table, Globals,
// and for a case the tile-staged kernel can take, its tensor maps.
CaseLayout case_layout(const BatchImpl* I, size_t elem, int nx, int ny, int nz) {
  CaseLayout L;
  const size_t N = (size_t)nx * ny * nz;
  L.stride = align_up(N, 256 / elem);
  L.buf = L.stride * I->Q * elem;
  L.flags = align_up(N * sizeof(flag_t), 256);
  L.zone = align_up((size_t)(1 << (16 - I->zone_shift)) * I->NZS * I->real_size, 256);
  L.glob = align_up(I->NG * sizeof(double), 256);
  L.maps = staged_rows(I, elem, nx, ny) ? align_up(sizeof(BatchTmaMaps), 256) : 0;
  L.total = 2 * L.buf + L.flags + L.zone + L.glob + L.maps;
  return L;
}

// Per case (iterations done, left), then (error word of the staging waits, 0).
__global__ void k_batch_status(const BatchCase* cases, int n, const int* err, int2* status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) status[c] = make_int2(cases[c].counter, cases[c].remaining);
  else if (c == n) status[n] = make_int2(*err, 0);
}

}  // namespace

struct tclb_batch {
  int model, precision, storage, device;
  const BatchImpl* I;
  size_t elem, budget, used = 0;
  int max_cases;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  BatchCase* d_cases = nullptr;
  int2* d_status = nullptr;
  int2* h_status = nullptr;  // pinned
  int* d_ntiles = nullptr;   // [0] tiles of the cases not staged, [1] all tiles, [2] staged tiles
  int* d_err = nullptr;      // staging wait ran out
  BatchTile* d_tiles = nullptr;
  BatchTmaTile* d_ttiles = nullptr;
  size_t tiles_cap = 0, ttiles_cap = 0;
  std::vector<BatchCase> cases;
  std::vector<size_t> bytes;
  std::vector<char> used_slot;
  bool tiles_dirty = true;
  int ntiles = 0, nplain = 0, nttiles = 0;
  int bx = 128, by = 2, K = 16, grid_blocks = 0, user_grid = 0;
  int sms = 148;   // multiprocessors of the device
  int tile_h = 0;  // height of the tiles in the table
  int tma_grid = -1;  // resident blocks of the tile-staged kernel (-1: not yet asked)
  // Settings of the staged group: for models with the packed collision the
  // tile-staged launch takes its settings as kernel parameters, so only the
  // cases with these settings are staged (the others take the pair kernel).
  // Chosen when the tile table is rebuilt: kept while a live case has them.
  std::vector<double> group;
  bool staging = false;  // the staged kernel runs (update_staging)
  int status_n = -1;  // cases in the status read back by the last step (its error word follows)
  cudaGraphExec_t graph = nullptr;
  cudaGraph_t graph_src = nullptr;          // kept: its nodes address the instantiated graph
  std::vector<cudaGraphNode_t> plain_nodes;  // one-block-per-tile plain launches
  std::vector<cudaGraphNode_t> glob_nodes;   // the Globals launch
  int graph_grid[2] = {0, 0};                // their grids in the instantiated graph
  int graph_key[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
  int paths = TCLB_LAUNCH_PAIRS | TCLB_LAUNCH_TMA | TCLB_BATCH_ADAPTIVE;  // tclb_batch_set_paths
};

namespace {

int upload_case(tclb_batch* B, int slot) {
  BCK(cudaMemcpyAsync(B->d_cases + slot, &B->cases[slot], sizeof(BatchCase), cudaMemcpyHostToDevice, B->stream));
  return TCLB_OK;
}

// Plain launches take the pair kernel: 16-bit storage, pairs enabled, one
// block per tile, tile width a multiple of 64 and the block (bx / 2, by)
// within the pair kernel's launch bounds.
bool pair_form(const tclb_batch* B) {
  return (B->paths & TCLB_LAUNCH_PAIRS) && B->user_grid == 0 && B->I->pair_threads > 0 && B->bx % 64 == 0 &&
         B->bx / 2 <= B->I->pair_threads;
}

bool in_group(const tclb_batch* B, const BatchCase& C) {
  if (!B->I->group_staging) return true;
  if ((int)B->group.size() != B->I->NSET) return false;
  for (int i = 0; i < B->I->NSET; i++)
    if (C.s[i] != B->group[i]) return false;
  return true;
}

// The case could take the tile-staged kernel: staging enabled, one block per
// tile, the case fits it (tensor maps were made) and belongs to the group.
bool stageable(const tclb_batch* B, const BatchCase& C) {
  return (B->paths & TCLB_LAUNCH_TMA) && B->user_grid == 0 && C.tma_rows > 0 && B->tma_grid > 0 && in_group(B, C);
}

// Plain launches of this case take the tile-staged kernel (see update_staging).
bool staged(const tclb_batch* B, const BatchCase& C) { return B->staging && stageable(B, C); }

bool live(const tclb_batch* B, size_t s) {
  return B->used_slot[s] && B->cases[s].active && B->h_status[s].y > 0;  // finished cases get no tiles
}

// Tile height: the set by, halved (down to the block's thread rows) while
// the live cases would give fewer tiles than two waves of resident blocks --
// a few small cases alone run as many short tiles, not a few long ones.
int tile_height(const tclb_batch* B) {
  int floor_h = block_rows(B->bx, B->by, 256);
  if (pair_form(B)) floor_h = std::max(floor_h, block_rows(B->bx / 2, B->by, B->I->pair_threads));
  if (!(B->paths & TCLB_BATCH_ADAPTIVE)) return B->by;
  int per_sm = B->I->blocks_per_sm(B->bx * floor_h);
  if (per_sm < 1) per_sm = std::max(1, 2048 / (B->bx * floor_h));
  const size_t want = (size_t)2 * B->sms * per_sm;
  auto count = [&](int h) {
    size_t n = 0;
    for (size_t s = 0; s < B->cases.size(); s++) {
      const BatchCase& C = B->cases[s];
      if (live(B, s) && !staged(B, C)) n += (size_t)C.nz * ((C.ny + h - 1) / h) * ((C.nx + B->bx - 1) / B->bx);
    }
    return n;
  };
  int h = B->by;
  while (h > floor_h && count(h) < want) h = std::max(floor_h, h / 2);
  return h;
}

// Grow a device table (pool memory) to hold n entries; a move forces a recapture.
template <class E>
int reserve(tclb_batch* B, E*& d, size_t& cap, size_t n) {
  if (n <= cap) return TCLB_OK;
  if (d) BCK(cudaFreeAsync(d, B->stream));
  cap = std::max(n, cap * 2);
  BCK(cudaMallocFromPoolAsync((void**)&d, cap * sizeof(E), B->pool, B->stream));
  B->graph_key[0] = -1;
  return TCLB_OK;
}

// The tile tables: bx x h tiles of the cases not staged, then those of the
// staged cases (the Globals launch covers both), and the staged cases'
// R-row tiles.
// The staged group: kept while a live case that fits the tile-staged kernel
// has its settings, else the settings of the first such case.
void choose_group(tclb_batch* B) {
  if (!B->I->group_staging) return;
  const BatchCase* first = nullptr;
  for (size_t s = 0; s < B->cases.size(); s++) {
    const BatchCase& C = B->cases[s];
    if (!live(B, s) || C.tma_rows == 0) continue;
    if (in_group(B, C)) return;
    if (!first) first = &C;
  }
  if (first) {
    B->group.assign(first->s, first->s + B->I->NSET);
    B->tiles_dirty = true;
  }
}

// Staging on while the stageable live cases give at least 8 tiles per
// resident block of the persistent staged kernel (with TCLB_BATCH_ADAPTIVE):
// with fewer, its per-launch pipeline start costs more than it saves.
void update_staging(tclb_batch* B) {
  if (B->tma_grid < 0) B->tma_grid = B->I->tma_grid(B->sms);
  choose_group(B);
  size_t n = 0;
  for (size_t s = 0; s < B->cases.size(); s++) {
    const BatchCase& C = B->cases[s];
    if (live(B, s) && stageable(B, C)) n += (size_t)C.nz * (C.ny / C.tma_rows);
  }
  const bool on = n > 0 && (!(B->paths & TCLB_BATCH_ADAPTIVE) || n >= (size_t)8 * B->tma_grid);
  if (on != B->staging) B->tiles_dirty = true;
  B->staging = on;
}

int rebuild_tiles(tclb_batch* B) {
  update_staging(B);
  std::vector<BatchTile> t;
  std::vector<BatchTmaTile> tt;
  const int h = tile_height(B);
  for (int pass = 0; pass < 2; pass++) {  // the cases not staged, then the staged ones
    for (size_t s = 0; s < B->cases.size(); s++) {
      const BatchCase& C = B->cases[s];
      if (!live(B, s) || staged(B, C) != (pass == 1)) continue;
      for (int z = 0; z < C.nz; z++)
        for (int y = 0; y < C.ny; y += h)
          for (int x = 0; x < C.nx; x += B->bx) t.push_back({(int)s, x, y, z, h});
      if (pass == 1)
        for (int z = 0; z < C.nz; z++)
          for (int y = 0; y < C.ny; y += C.tma_rows) tt.push_back({(int)s, z, y});
    }
    if (pass == 0) B->nplain = (int)t.size();
  }
  B->tile_h = h;
  int rc;
  if ((rc = reserve(B, B->d_tiles, B->tiles_cap, t.size())) || (rc = reserve(B, B->d_ttiles, B->ttiles_cap, tt.size())))
    return rc;
  B->ntiles = (int)t.size();
  B->nttiles = (int)tt.size();
  if (!t.empty())
    BCK(cudaMemcpyAsync(B->d_tiles, t.data(), t.size() * sizeof(BatchTile), cudaMemcpyHostToDevice, B->stream));
  if (!tt.empty())
    BCK(cudaMemcpyAsync(B->d_ttiles, tt.data(), tt.size() * sizeof(BatchTmaTile), cudaMemcpyHostToDevice,
                        B->stream));
  const int n[3] = {B->nplain, B->ntiles, B->nttiles};
  BCK(cudaMemcpyAsync(B->d_ntiles, n, sizeof(n), cudaMemcpyHostToDevice, B->stream));
  BCK(cudaStreamSynchronize(B->stream));  // the host vectors die here
  B->tiles_dirty = false;
  return TCLB_OK;
}

// One block per tile: the grid of the plain launches is the count of tiles
// of the cases not staged, that of the Globals launch the count of all tiles.
// When only those change, the kernel nodes of the instantiated graph get the
// new grids in place (no recapture).
int update_graph_grid(tclb_batch* B) {
  if (B->user_grid != 0) return TCLB_OK;
  const int grid[2] = {std::max(1, B->nplain), std::max(1, B->ntiles)};
  for (int w = 0; w < 2; w++) {
    if (grid[w] == B->graph_grid[w]) continue;
    for (cudaGraphNode_t node : (w ? B->glob_nodes : B->plain_nodes)) {
      cudaKernelNodeParams p;
      BCK(cudaGraphKernelNodeGetParams(node, &p));
      p.gridDim = dim3(grid[w]);
      BCK(cudaGraphExecKernelNodeSetParams(B->graph, node, &p));
    }
    B->graph_grid[w] = grid[w];
  }
  return TCLB_OK;
}

int ensure_graph(tclb_batch* B) {
  const int has_tma = B->nttiles > 0;
  // the staged group's settings are captured as kernel parameters
  const int group_hash = (int)std::hash<std::string>()(
      std::string(reinterpret_cast<const char*>(B->group.data()), B->group.size() * sizeof(double)));
  const int key[8] = {B->bx, B->by, B->K, (int)B->cases.size(), B->user_grid, B->paths, has_tma, group_hash};
  if (B->graph && std::equal(key, key + 8, B->graph_key)) return update_graph_grid(B);
  if (B->graph) {
    cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
  }
  if (B->graph_src) {
    cudaGraphDestroy(B->graph_src);
    B->graph_src = nullptr;
  }
  B->plain_nodes.clear();
  B->glob_nodes.clear();
  const int threads = B->bx * block_rows(B->bx, B->by, 256);
  int per_sm = B->I->blocks_per_sm(threads);
  if (per_sm < 1) per_sm = std::max(1, 2048 / threads);
  // grid_blocks 0 (default): one block per live tile; > 0: a persistent grid
  // of that size walking the tiles; < 0: persistent, SMs x resident blocks.
  const bool per_tile = B->user_grid == 0;
  B->grid_blocks = per_tile ? std::max(1, B->nplain) : (B->user_grid > 0 ? B->user_grid : B->sms * per_sm);
  const int grid_all = per_tile ? std::max(1, B->ntiles) : B->grid_blocks;
  const int form = !per_tile ? FORM_PERSISTENT : (pair_form(B) ? FORM_PAIR : FORM_TILE);
  const LaunchTables L = {B->d_cases, B->d_tiles, B->d_ntiles, B->d_ttiles, B->d_ntiles + 2, B->d_err};
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  const int n = (int)B->cases.size();
  B->I->clear(B->d_cases, n, B->K, B->stream);
  for (int k = 0; k < B->K; k++)
    B->I->iterate(L, k, B->K, dim3(B->grid_blocks), dim3(grid_all), has_tma ? B->tma_grid : 0,
                  B->group.empty() ? nullptr : B->group.data(), B->bx, B->by, form,
                  (B->paths & TCLB_BATCH_GLOBALS_AT_END) != 0, B->stream);
  if (n > 0) {
    k_batch_advance<<<(n + 127) / 128, 128, 0, B->stream>>>(B->d_cases, n, B->K);
    k_batch_status<<<(n + 128) / 128, 128, 0, B->stream>>>(B->d_cases, n, B->d_err, B->d_status);
  }
  cudaError_t e = cudaStreamEndCapture(B->stream, &g);
  if (e != cudaSuccess) return bfail(TCLB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&B->graph, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return bfail(TCLB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  B->graph_src = g;
  if (per_tile) {  // remember the one-block-per-tile launches, to resize their grids later
    size_t count = 0;
    BCK(cudaGraphGetNodes(g, nullptr, &count));
    std::vector<cudaGraphNode_t> nodes(count);
    BCK(cudaGraphGetNodes(g, nodes.data(), &count));
    const void* f0 = B->I->tile_kernel(0);
    const void* f1 = B->I->tile_kernel(1);
    const void* f2 = B->I->tile_kernel(2);
    for (cudaGraphNode_t node : nodes) {
      cudaGraphNodeType type;
      BCK(cudaGraphNodeGetType(node, &type));
      if (type != cudaGraphNodeTypeKernel) continue;
      cudaKernelNodeParams p;
      BCK(cudaGraphKernelNodeGetParams(node, &p));
      if (p.func == f0 || (f2 && p.func == f2)) B->plain_nodes.push_back(node);
      else if (p.func == f1) B->glob_nodes.push_back(node);
    }
  }
  B->graph_grid[0] = B->grid_blocks;
  B->graph_grid[1] = grid_all;
  std::copy(key, key + 8, B->graph_key);
  return TCLB_OK;
}

#define CHECK_B(b) \
  if (!(b)) return bfail(TCLB_ERR_ARG, "null batch handle")

}  // namespace

namespace {

// Lay out case `slot` in its allocation p, upload its tables and fields,
// and write its descriptor to the device (the caller registers it).
int fill_case(tclb_batch* B, int slot, char* p, const CaseLayout& L, const ModelTable* T, int nzones, int nx,
              int ny, int nz, const uint16_t* flags, const double* settings, const double* zone_settings,
              int zone_rows, int niter) {
  BatchCase C;
  std::memset(&C, 0, sizeof(C));
  C.buf[0] = p;
  C.buf[1] = p + L.buf;
  C.flags = reinterpret_cast<flag_t*>(p + 2 * L.buf);
  C.zone = p + 2 * L.buf + L.flags;
  C.glob = reinterpret_cast<double*>(p + 2 * L.buf + L.flags + L.zone);
  C.stride = L.stride;
  C.nx = nx;
  C.ny = ny;
  C.nz = nz;
  C.counter = 0;
  C.remaining = niter;
  C.active = 1;
  C.glob_end = (B->paths & TCLB_BATCH_GLOBALS_AT_END) ? 1 : 0;
  BatchTmaMaps maps;  // host copy of the tensor maps, uploaded below
  if (L.maps) {
    const int R = staged_rows(B->I, B->elem, nx, ny);
    bool ok = true;
    for (int b = 0; b < 2 && ok; b++)
      ok = encode_tile_maps(C.buf[b], C.flags, nx, ny, nz, B->I->Q, L.stride, R, &maps.rows[b], &maps.row1[b],
                            &maps.flags);
    if (ok) {  // otherwise the case runs the register kernels
      C.tma_rows = R;
      C.maps = reinterpret_cast<const BatchTmaMaps*>(p + 2 * L.buf + L.flags + L.zone + L.glob);
      BCK(cudaMemcpyAsync(const_cast<BatchTmaMaps*>(C.maps), &maps, sizeof(maps), cudaMemcpyHostToDevice,
                          B->stream));
    }
  }
  for (int i = 0; i < T->nsettings && i < BATCH_MAX_SET; i++) C.s[i] = settings[i];
  B->I->derive(C);
  // zonal table: default values, then the caller's rows (zone 0.. zone_rows-1)
  const int nzs = T->nzonesettings;
  std::vector<double> zt((size_t)nzones * nzs);
  for (int z = 0; z < nzones; z++)
    for (int s = 0; s < nzs; s++) zt[(size_t)z * nzs + s] = T->zone_setting_defaults[s];
  for (int z = 0; z < zone_rows; z++)
    for (int s = 0; s < nzs; s++) zt[(size_t)z * nzs + s] = zone_settings[(size_t)z * nzs + s];
  if (B->precision == TCLB_FP64) {
    BCK(cudaMemcpyAsync(const_cast<void*>(C.zone), zt.data(), zt.size() * 8, cudaMemcpyHostToDevice, B->stream));
  } else {
    std::vector<float> zf(zt.begin(), zt.end());
    BCK(cudaMemcpyAsync(const_cast<void*>(C.zone), zf.data(), zf.size() * 4, cudaMemcpyHostToDevice, B->stream));
    BCK(cudaStreamSynchronize(B->stream));
  }
  BCK(cudaMemcpyAsync(const_cast<flag_t*>(C.flags), flags, (size_t)nx * ny * nz * sizeof(flag_t),
                      cudaMemcpyHostToDevice, B->stream));
  BCK(cudaMemsetAsync(C.glob, 0, B->I->NG * sizeof(double), B->stream));
  B->I->init(C, C.buf[0], B->stream, 32, 4);
  BCK(cudaGetLastError());
  B->cases[slot] = C;
  int rc = upload_case(B, slot);
  if (rc) return rc;
  BCK(cudaStreamSynchronize(B->stream));
  return TCLB_OK;
}

}  // namespace

extern "C" {

const char* tclb_batch_last_error(void) { return g_batch_err.c_str(); }

size_t tclb_batch_case_bytes(int model, int precision, int storage, int nx, int ny, int nz) {
  const BatchImpl* I = bimpl(model, precision, storage);
  if (!I || nx < 1 || ny < 1 || nz < 1) return 0;
  return case_layout(I, elem_size(precision, storage), nx, ny, nz).total;
}

int tclb_batch_create(tclb_batch_h* out, int model, int precision, int storage, size_t budget_bytes, int max_cases) {
  if (!out) return bfail(TCLB_ERR_ARG, "null output handle");
  *out = nullptr;
  const BatchImpl* I = bimpl(model, precision, storage);
  if (!I) return bfail(TCLB_ERR_ARG, "unsupported model/precision/storage");
  if (max_cases < 1 || max_cases > (1 << 20)) return bfail(TCLB_ERR_ARG, "max_cases out of range");
  tclb_batch* B = new tclb_batch();
  B->model = model;
  B->precision = precision;
  B->storage = storage;
  B->I = I;
  B->elem = elem_size(precision, storage);
  B->budget = budget_bytes;
  B->max_cases = max_cases;
  cudaGetDevice(&B->device);
  cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, B->device);
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = B->device;
  cudaError_t e = cudaMemPoolCreate(&B->pool, &props);
  if (e == cudaSuccess) {
    uint64_t thr = UINT64_MAX;  // keep freed memory in the pool for the next admissions
    e = cudaMemPoolSetAttribute(B->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_cases, sizeof(BatchCase) * max_cases);
  if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_status, sizeof(int2) * (max_cases + 1));
  if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_ntiles, 3 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(B->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&B->h_status, sizeof(int2) * (max_cases + 1));
  if (e == cudaSuccess) std::memset(B->h_status, 0, sizeof(int2) * (max_cases + 1));
  if (e == cudaSuccess) e = cudaMemset(B->d_cases, 0, sizeof(BatchCase) * max_cases);
  if (e == cudaSuccess) e = cudaMemset(B->d_ntiles, 0, 3 * sizeof(int));
  if (e != cudaSuccess) {
    tclb_batch_destroy(B);
    return bfail(TCLB_ERR_CUDA, std::string("batch create: ") + cudaGetErrorString(e));
  }
  *out = B;
  return TCLB_OK;
}

int tclb_batch_destroy(tclb_batch_h B) {
  CHECK_B(B);
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->graph) cudaGraphExecDestroy(B->graph);
  if (B->graph_src) cudaGraphDestroy(B->graph_src);
  for (size_t s = 0; s < B->cases.size(); s++)
    if (B->used_slot[s]) cudaFreeAsync(B->cases[s].buf[0], B->stream);
  if (B->d_tiles) cudaFreeAsync(B->d_tiles, B->stream);
  if (B->d_ttiles) cudaFreeAsync(B->d_ttiles, B->stream);
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->d_cases) cudaFree(B->d_cases);
  if (B->d_status) cudaFree(B->d_status);
  if (B->d_ntiles) cudaFree(B->d_ntiles);
  if (B->d_err) cudaFree(B->d_err);
  if (B->h_status) cudaFreeHost(B->h_status);
  if (B->pool) cudaMemPoolDestroy(B->pool);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return TCLB_OK;
}

int tclb_batch_add_case(tclb_batch_h B, int nx, int ny, int nz, const uint16_t* flags, const double* settings,
                        const double* zone_settings, int zone_rows, int niter, int* case_id) {
  CHECK_B(B);
  const ModelTable* T = model_table(B->model);
  if (nx < 1 || ny < 1 || nz < 1 || !flags || !settings || !case_id || niter < 0)
    return bfail(TCLB_ERR_ARG, "bad case arguments");
  if (T->dim == 2 && nz != 1) return bfail(TCLB_ERR_ARG, "2D model needs nz == 1");
  if ((size_t)nx * ny * nz >= ((size_t)1 << 31)) return bfail(TCLB_ERR_ARG, "case above 2^31 nodes");
  const int nzones = 1 << (16 - B->I->zone_shift);
  if (zone_rows < 0 || zone_rows > nzones || (zone_rows > 0 && !zone_settings))
    return bfail(TCLB_ERR_ARG, "zone rows out of range");
  const CaseLayout L = case_layout(B->I, B->elem, nx, ny, nz);
  if (B->used + L.total > B->budget) return bfail(TCLB_ERR_MEMORY, "admission refused: memory budget exceeded");
  int slot = -1;
  for (size_t s = 0; s < B->cases.size(); s++)
    if (!B->used_slot[s]) { slot = (int)s; break; }
  if (slot < 0) {
    if ((int)B->cases.size() >= B->max_cases) return bfail(TCLB_ERR_MEMORY, "admission refused: no free case slot");
    slot = (int)B->cases.size();
    B->cases.push_back(BatchCase());
    B->bytes.push_back(0);
    B->used_slot.push_back(0);
  }
  char* p = nullptr;
  BCK(cudaMallocFromPoolAsync((void**)&p, L.total, B->pool, B->stream));
  const int rc = fill_case(B, slot, p, L, T, nzones, nx, ny, nz, flags, settings, zone_settings, zone_rows, niter);
  if (rc) {  // the allocation goes back to the pool; the slot stays free
    cudaFreeAsync(p, B->stream);
    std::memset(&B->cases[slot], 0, sizeof(BatchCase));
    return rc;
  }
  B->bytes[slot] = L.total;
  B->used_slot[slot] = 1;
  B->used += L.total;
  B->h_status[slot] = make_int2(0, niter);
  B->tiles_dirty = true;
  *case_id = slot;
  return TCLB_OK;
}

int tclb_batch_reserve(tclb_batch_h B, size_t bytes) {
  CHECK_B(B);
  if (bytes > B->budget) return bfail(TCLB_ERR_ARG, "reserve: more than the batch's budget");
  constexpr size_t BLOCK = (size_t)1 << 31;
  std::vector<void*> blocks;
  cudaError_t e = cudaSuccess;
  for (size_t done = 0; done < bytes && e == cudaSuccess; done += BLOCK) {
    void* p = nullptr;
    e = cudaMallocFromPoolAsync(&p, std::min(BLOCK, bytes - done), B->pool, B->stream);
    if (e == cudaSuccess) blocks.push_back(p);
  }
  for (void* p : blocks) cudaFreeAsync(p, B->stream);  // back to the pool, which keeps them
  const cudaError_t s = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return bfail(TCLB_ERR_MEMORY, std::string("reserve: ") + cudaGetErrorString(e));
  }
  BCK(s);
  return TCLB_OK;
}

int tclb_batch_remove_case(tclb_batch_h B, int id) {
  CHECK_B(B);
  if (id < 0 || id >= (int)B->cases.size() || !B->used_slot[id]) return bfail(TCLB_ERR_ARG, "unknown case");
  B->cases[id].active = 0;
  int rc = upload_case(B, id);
  if (rc) return rc;
  BCK(cudaFreeAsync(B->cases[id].buf[0], B->stream));
  B->used -= B->bytes[id];
  B->bytes[id] = 0;
  B->used_slot[id] = 0;
  B->tiles_dirty = true;
  return TCLB_OK;
}

int tclb_batch_set_priority(tclb_batch_h B, int high) {
  CHECK_B(B);
  int least = 0, greatest = 0;
  BCK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  BCK(cudaStreamSynchronize(B->stream));  // pool allocations made on the old stream are complete
  cudaStream_t s = nullptr;
  BCK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high ? greatest : least));
  cudaStreamDestroy(B->stream);
  B->stream = s;
  return TCLB_OK;
}

int tclb_batch_set_launch(tclb_batch_h B, int bx, int by, int iters_per_launch, int grid_blocks) {
  CHECK_B(B);
  if (bx < 32 || bx % 32 || bx > 256 || by < 1 || by > 256 || iters_per_launch < 1 || iters_per_launch > 4096)
    return bfail(TCLB_ERR_ARG, "bad launch shape");
  B->tiles_dirty = true;  // the shape and the grid form decide the tables
  B->bx = bx;
  B->by = by;
  B->K = iters_per_launch;
  B->user_grid = grid_blocks;
  B->graph_key[0] = -1;
  return TCLB_OK;
}

int tclb_batch_set_paths(tclb_batch_h B, int flags) {
  CHECK_B(B);
  if (flags & ~(TCLB_LAUNCH_PAIRS | TCLB_LAUNCH_TMA | TCLB_BATCH_ADAPTIVE | TCLB_BATCH_GLOBALS_AT_END))
    return bfail(TCLB_ERR_ARG, "unknown path flags");
  if (flags != B->paths) B->tiles_dirty = true;
  if ((flags ^ B->paths) & TCLB_BATCH_GLOBALS_AT_END) {  // the case descriptors carry the Globals mode
    BCK(cudaStreamSynchronize(B->stream));
    for (size_t s = 0; s < B->cases.size(); s++) {
      if (!B->used_slot[s]) continue;
      B->cases[s].glob_end = (flags & TCLB_BATCH_GLOBALS_AT_END) ? 1 : 0;
      int rc = upload_case(B, (int)s);
      if (rc) return rc;
    }
    BCK(cudaStreamSynchronize(B->stream));
  }
  B->paths = flags;
  B->graph_key[0] = -1;
  return TCLB_OK;
}

int tclb_batch_get_paths(tclb_batch_h B, int* flags) {
  CHECK_B(B);
  update_staging(B);
  bool any_staged = false;
  for (size_t s = 0; s < B->cases.size(); s++) any_staged |= live(B, s) && staged(B, B->cases[s]);
  if (flags)
    *flags = (pair_form(B) ? TCLB_LAUNCH_PAIRS : 0) | (any_staged ? TCLB_LAUNCH_TMA : 0) |
             (B->paths & (TCLB_BATCH_ADAPTIVE | TCLB_BATCH_GLOBALS_AT_END));
  return TCLB_OK;
}

int tclb_batch_get_launch(tclb_batch_h B, int* bx, int* by, int* iters_per_launch) {
  CHECK_B(B);
  if (bx) *bx = B->bx;
  if (by) *by = B->by;
  if (iters_per_launch) *iters_per_launch = B->K;
  return TCLB_OK;
}

// One replay: up to K iterations of every active case with iterations left,
// Globals of each case's last iteration in the replay, then the counters.
int tclb_batch_step(tclb_batch_h B) {
  CHECK_B(B);
  int rc;
  if (B->tiles_dirty && (rc = rebuild_tiles(B))) return rc;
  if (B->cases.empty() || B->ntiles == 0) return TCLB_OK;
  if ((rc = ensure_graph(B))) return rc;
  BCK(cudaGraphLaunch(B->graph, B->stream));
  B->status_n = (int)B->cases.size();
  BCK(cudaMemcpyAsync(B->h_status, B->d_status, sizeof(int2) * (B->status_n + 1), cudaMemcpyDeviceToHost,
                      B->stream));
  return TCLB_OK;
}

int tclb_batch_done(tclb_batch_h B) {
  if (!B) return bfail(TCLB_ERR_ARG, "null batch handle");
  const cudaError_t e = cudaStreamQuery(B->stream);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  return bfail(TCLB_ERR_CUDA, std::string("stream query: ") + cudaGetErrorString(e));
}

int tclb_batch_sync(tclb_batch_h B) {
  CHECK_B(B);
  BCK(cudaStreamSynchronize(B->stream));
  if (B->status_n >= 0 && B->h_status[B->status_n].x != 0) {  // a staging wait ran out
    B->h_status[B->status_n].x = 0;
    BCK(cudaMemsetAsync(B->d_err, 0, sizeof(int), B->stream));
    BCK(cudaStreamSynchronize(B->stream));
    return bfail(TCLB_ERR_CUDA, "tile pipeline: a wait for staged tiles ran out; the batch state is not valid");
  }
  // cases that finished in the last step leave the tile table
  for (size_t s = 0; s < B->cases.size(); s++)
    if (B->used_slot[s] && B->cases[s].active && B->h_status[s].y <= 0 && B->cases[s].remaining > 0) {
      B->cases[s].remaining = 0;
      B->tiles_dirty = true;
    }
  return TCLB_OK;
}

// After tclb_batch_sync: iterations done and left of a case, as of the last step.
int tclb_batch_poll(tclb_batch_h B, int id, long long* iterations_done, int* remaining) {
  CHECK_B(B);
  if (id < 0 || id >= (int)B->cases.size() || !B->used_slot[id]) return bfail(TCLB_ERR_ARG, "unknown case");
  if (iterations_done) *iterations_done = B->h_status[id].x;
  if (remaining) *remaining = B->h_status[id].y;
  return TCLB_OK;
}

int tclb_batch_get_globals(tclb_batch_h B, int id, double* out) {
  CHECK_B(B);
  if (id < 0 || id >= (int)B->cases.size() || !B->used_slot[id] || !out) return bfail(TCLB_ERR_ARG, "unknown case");
  BCK(cudaMemcpyAsync(out, B->cases[id].glob, B->I->NG * sizeof(double), cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  return TCLB_OK;
}

// Quantity q of the whole case (after sync), real_t values as tclb_get_quantity.
int tclb_batch_get_quantity(tclb_batch_h B, int id, int q, void* out, double scale) {
  CHECK_B(B);
  const ModelTable* T = model_table(B->model);
  if (id < 0 || id >= (int)B->cases.size() || !B->used_slot[id] || !out) return bfail(TCLB_ERR_ARG, "unknown case");
  if (q < 0 || q >= T->nquantities) return bfail(TCLB_ERR_ARG, "quantity index out of range");
  BCK(cudaStreamSynchronize(B->stream));
  const BatchCase& C = B->cases[id];
  const int vec = T->quantity_vector[q];
  const size_t bytes = (size_t)C.nx * C.ny * C.nz * (vec ? 3 : 1) * B->I->real_size;
  void* tmp = nullptr;
  BCK(cudaMallocFromPoolAsync(&tmp, bytes, B->pool, B->stream));
  const int parity = B->h_status[id].x & 1;
  B->I->quantity(C, parity, q, vec, scale, tmp, B->stream);
  BCK(cudaGetLastError());
  BCK(cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToHost, B->stream));
  BCK(cudaFreeAsync(tmp, B->stream));
  BCK(cudaStreamSynchronize(B->stream));
  return TCLB_OK;
}

int tclb_batch_info(tclb_batch_h B, int* ncases_active, int* ntiles, size_t* used_bytes, size_t* budget_bytes) {
  CHECK_B(B);
  if (ncases_active) {
    int n = 0;
    for (size_t s = 0; s < B->cases.size(); s++) n += B->used_slot[s] && B->cases[s].active;
    *ncases_active = n;
  }
  if (ntiles) *ntiles = B->ntiles;
  if (used_bytes) *used_bytes = B->used;
  if (budget_bytes) *budget_bytes = B->budget;
  return TCLB_OK;
}

// Total node updates a step will perform (sum over active cases of
// nodes * min(K, remaining)), as of the last status read-back.
long long tclb_batch_pending_updates(tclb_batch_h B) {
  if (!B) return -1;
  long long u = 0;
  for (size_t s = 0; s < B->cases.size(); s++) {
    if (!B->used_slot[s] || !B->cases[s].active) continue;
    const long long n = (long long)B->cases[s].nx * B->cases[s].ny * B->cases[s].nz;
    u += n * std::min(B->K, B->h_status[s].y);
  }
  return u;
}

}  // extern "C"
