// Batched lattices: many independent cases of one model advanced by one
// launch per iteration, K iterations per CUDA-graph replay. New API (no
// counterpart in the reference, which runs one lattice per process).
//
// Memory: each case is one allocation from a stream-ordered CUDA memory pool
// owned by the batch (two snapshots, node types, zonal settings, Globals), so
// admitting and retiring cases never synchronises the device. A byte budget
// bounds the sum of case footprints; admission beyond it is refused.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
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

struct BatchImpl {
  // launch k of K over tiles of bx x by nodes; FORM_PAIR runs the pair kernel
  // on plain launches (bx / 2 threads per row) and the one-tile kernel on the
  // Globals launch (bx threads per row)
  void (*iterate)(const BatchCase*, const BatchTile*, const int*, int, int, dim3, int bx, int by, int form,
                  cudaStream_t);
  void (*clear)(BatchCase*, int, cudaStream_t);
  void (*init)(const BatchCase&, const void* dst, cudaStream_t, int bx, int by);
  void (*quantity)(const BatchCase&, int parity, int q, int vec, double scale, void* out, cudaStream_t);
  int (*blocks_per_sm)(int threads);
  const void* (*tile_kernel)(int which);  // 0 one-tile plain, 1 one-tile Globals, 2 pair
  int pair_threads;                        // block-size limit of the pair kernel; 0: no pair kernel
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
  static void iterate(const BatchCase* c, const BatchTile* t, const int* n, int k, int K, dim3 g, int bx, int by,
                      int form, cudaStream_t s) {
    const dim3 b(bx, block_rows(bx, by, 256));
    if constexpr (pairs) {
      if (form == FORM_PAIR && k != K - 1) {
        const dim3 bp(bx / 2, block_rows(bx / 2, by, M::PAIR_THREADS));
        k_iterate_batch_pair<M, R, St><<<g, bp, 0, s>>>(c, t, n, k, K);
        return;
      }
    }
    if (form != FORM_PERSISTENT) {
      if (k == K - 1) k_iterate_batch_tile<M, R, St, true><<<g, b, 0, s>>>(c, t, n, k, K);
      else k_iterate_batch_tile<M, R, St, false><<<g, b, 0, s>>>(c, t, n, k, K);
    } else {
      if (k == K - 1) k_iterate_batch<M, R, St, true><<<g, b, 0, s>>>(c, t, n, k, K);
      else k_iterate_batch<M, R, St, false><<<g, b, 0, s>>>(c, t, n, k, K);
    }
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
  static void clear(BatchCase* c, int n, cudaStream_t s) {
    if (n > 0) k_batch_clear_globals<M::NG><<<n, 32, 0, s>>>(c, n);
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
  static const BatchImpl* get() {
    static const BatchImpl impl = {iterate,     clear, init, quantity, blocks_per_sm, tile_kernel,
                                   pairs ? M::PAIR_THREADS : 0, sizeof(R), M::Q, M::NG, M::NSET, M::NZS,
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
  size_t stride, buf, flags, zone, glob, total;
};

CaseLayout case_layout(const BatchImpl* I, size_t elem, int nx, int ny, int nz) {
  CaseLayout L;
  const size_t N = (size_t)nx * ny * nz;
  L.stride = align_up(N, 256 / elem);
  L.buf = L.stride * I->Q * elem;
  L.flags = align_up(N * sizeof(flag_t), 256);
  L.zone = align_up((size_t)(1 << (16 - I->zone_shift)) * I->NZS * I->real_size, 256);
  L.glob = align_up(I->NG * sizeof(double), 256);
  L.total = 2 * L.buf + L.flags + L.zone + L.glob;
  return L;
}

__global__ void k_batch_status(const BatchCase* cases, int n, int2* status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) status[c] = make_int2(cases[c].counter, cases[c].remaining);
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
  int* d_ntiles = nullptr;
  BatchTile* d_tiles = nullptr;
  size_t tiles_cap = 0;
  std::vector<BatchCase> cases;
  std::vector<size_t> bytes;
  std::vector<char> used_slot;
  bool tiles_dirty = true;
  int ntiles = 0;
  int bx = 128, by = 2, K = 16, grid_blocks = 0, user_grid = 0;
  int sms = 148;   // multiprocessors of the device
  int tile_h = 0;  // height of the tiles in the table
  cudaGraphExec_t graph = nullptr;
  cudaGraph_t graph_src = nullptr;            // kept: its nodes address the instantiated graph
  std::vector<cudaGraphNode_t> iter_nodes;    // the K iteration launches (one block per tile)
  int graph_grid = 0;                         // their grid size in the instantiated graph
  int graph_key[6] = {-1, -1, -1, -1, -1, -1};
  int paths = TCLB_LAUNCH_PAIRS | TCLB_BATCH_SHORT_TILES;  // tclb_batch_set_paths
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

// Tile height: the set by, halved (down to the block's thread rows) while
// the live cases would give fewer tiles than two waves of resident blocks --
// a few small cases alone run as many short tiles, not a few long ones.
int tile_height(const tclb_batch* B) {
  int floor_h = block_rows(B->bx, B->by, 256);
  if (pair_form(B)) floor_h = std::max(floor_h, block_rows(B->bx / 2, B->by, B->I->pair_threads));
  if (!(B->paths & TCLB_BATCH_SHORT_TILES)) return B->by;
  int per_sm = B->I->blocks_per_sm(B->bx * floor_h);
  if (per_sm < 1) per_sm = std::max(1, 2048 / (B->bx * floor_h));
  const size_t want = (size_t)2 * B->sms * per_sm;
  auto count = [&](int h) {
    size_t n = 0;
    for (size_t s = 0; s < B->cases.size(); s++) {
      const BatchCase& C = B->cases[s];
      if (!B->used_slot[s] || !C.active || B->h_status[s].y <= 0) continue;
      n += (size_t)C.nz * ((C.ny + h - 1) / h) * ((C.nx + B->bx - 1) / B->bx);
    }
    return n;
  };
  int h = B->by;
  while (h > floor_h && count(h) < want) h = std::max(floor_h, h / 2);
  return h;
}

int rebuild_tiles(tclb_batch* B) {
  std::vector<BatchTile> t;
  const int h = tile_height(B);
  for (size_t s = 0; s < B->cases.size(); s++) {
    const BatchCase& C = B->cases[s];
    if (!B->used_slot[s] || !C.active || B->h_status[s].y <= 0) continue;  // finished cases get no tiles
    for (int z = 0; z < C.nz; z++)
      for (int y = 0; y < C.ny; y += h)
        for (int x = 0; x < C.nx; x += B->bx) t.push_back({(int)s, x, y, z, h});
  }
  B->tile_h = h;
  if (t.size() > B->tiles_cap) {
    if (B->d_tiles) BCK(cudaFreeAsync(B->d_tiles, B->stream));
    B->tiles_cap = std::max(t.size(), B->tiles_cap * 2);
    BCK(cudaMallocFromPoolAsync((void**)&B->d_tiles, B->tiles_cap * sizeof(BatchTile), B->pool, B->stream));
    B->graph_key[0] = -1;  // tile table moved: recapture
  }
  B->ntiles = (int)t.size();
  if (!t.empty())
    BCK(cudaMemcpyAsync(B->d_tiles, t.data(), t.size() * sizeof(BatchTile), cudaMemcpyHostToDevice, B->stream));
  BCK(cudaMemcpyAsync(B->d_ntiles, &B->ntiles, sizeof(int), cudaMemcpyHostToDevice, B->stream));
  BCK(cudaStreamSynchronize(B->stream));  // host vector t dies here
  B->tiles_dirty = false;
  return TCLB_OK;
}

// One block per tile: the iteration launches' grid is the live tile count.
// When only that changes, the K kernel nodes of the instantiated graph get
// the new grid in place (no recapture).
int update_graph_grid(tclb_batch* B) {
  const int grid = std::max(1, B->ntiles);
  if (B->user_grid != 0 || grid == B->graph_grid) return TCLB_OK;
  for (cudaGraphNode_t node : B->iter_nodes) {
    cudaKernelNodeParams p;
    BCK(cudaGraphKernelNodeGetParams(node, &p));
    p.gridDim = dim3(grid);
    BCK(cudaGraphExecKernelNodeSetParams(B->graph, node, &p));
  }
  B->graph_grid = grid;
  return TCLB_OK;
}

int ensure_graph(tclb_batch* B) {
  const int key[6] = {B->bx, B->by, B->K, (int)B->cases.size(), B->user_grid, B->paths};
  if (B->graph && std::equal(key, key + 6, B->graph_key)) return update_graph_grid(B);
  if (B->graph) {
    cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
  }
  if (B->graph_src) {
    cudaGraphDestroy(B->graph_src);
    B->graph_src = nullptr;
  }
  B->iter_nodes.clear();
  int dev = B->device, sms = 148, per_sm = 4;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = B->bx * block_rows(B->bx, B->by, 256);
  per_sm = B->I->blocks_per_sm(threads);
  if (per_sm < 1) per_sm = std::max(1, 2048 / threads);
  // grid_blocks 0 (default): one block per live tile; > 0: a persistent grid
  // of that size walking the tiles; < 0: persistent, SMs x resident blocks.
  const bool per_tile = B->user_grid == 0;
  B->grid_blocks = per_tile ? std::max(1, B->ntiles) : (B->user_grid > 0 ? B->user_grid : sms * per_sm);
  const int form = !per_tile ? FORM_PERSISTENT : (pair_form(B) ? FORM_PAIR : FORM_TILE);
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  const int n = (int)B->cases.size();
  B->I->clear(B->d_cases, n, B->stream);
  for (int k = 0; k < B->K; k++)
    B->I->iterate(B->d_cases, B->d_tiles, B->d_ntiles, k, B->K, dim3(B->grid_blocks), B->bx, B->by, form,
                  B->stream);
  if (n > 0) {
    k_batch_advance<<<(n + 127) / 128, 128, 0, B->stream>>>(B->d_cases, n, B->K);
    k_batch_status<<<(n + 127) / 128, 128, 0, B->stream>>>(B->d_cases, n, B->d_status);
  }
  cudaError_t e = cudaStreamEndCapture(B->stream, &g);
  if (e != cudaSuccess) return bfail(TCLB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&B->graph, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return bfail(TCLB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  B->graph_src = g;
  if (per_tile) {  // remember the iteration launches, to resize their grid later
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
      if (p.func == f0 || p.func == f1 || (f2 && p.func == f2)) B->iter_nodes.push_back(node);
    }
  }
  B->graph_grid = B->grid_blocks;
  std::copy(key, key + 6, B->graph_key);
  return TCLB_OK;
}

#define CHECK_B(b) \
  if (!(b)) return bfail(TCLB_ERR_ARG, "null batch handle")

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
  if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_status, sizeof(int2) * max_cases);
  if (e == cudaSuccess) e = cudaMalloc((void**)&B->d_ntiles, sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&B->h_status, sizeof(int2) * max_cases);
  if (e == cudaSuccess) e = cudaMemset(B->d_cases, 0, sizeof(BatchCase) * max_cases);
  if (e == cudaSuccess) e = cudaMemset(B->d_ntiles, 0, sizeof(int));
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
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->d_cases) cudaFree(B->d_cases);
  if (B->d_status) cudaFree(B->d_status);
  if (B->d_ntiles) cudaFree(B->d_ntiles);
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
  for (int i = 0; i < T->nsettings && i < BATCH_MAX_SET; i++) C.s[i] = settings[i];
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
  B->bytes[slot] = L.total;
  B->used_slot[slot] = 1;
  B->used += L.total;
  B->h_status[slot] = make_int2(0, niter);
  int rc = upload_case(B, slot);
  if (rc) return rc;
  BCK(cudaStreamSynchronize(B->stream));
  B->tiles_dirty = true;
  *case_id = slot;
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
  if (bx != B->bx || by != B->by) B->tiles_dirty = true;
  B->bx = bx;
  B->by = by;
  B->K = iters_per_launch;
  B->user_grid = grid_blocks;
  B->graph_key[0] = -1;
  return TCLB_OK;
}

int tclb_batch_set_paths(tclb_batch_h B, int flags) {
  CHECK_B(B);
  if (flags & ~(TCLB_LAUNCH_PAIRS | TCLB_BATCH_SHORT_TILES)) return bfail(TCLB_ERR_ARG, "unknown path flags");
  if ((flags ^ B->paths) & TCLB_BATCH_SHORT_TILES) B->tiles_dirty = true;
  B->paths = flags;
  B->graph_key[0] = -1;
  return TCLB_OK;
}

int tclb_batch_get_paths(tclb_batch_h B, int* flags) {
  CHECK_B(B);
  if (flags) *flags = (pair_form(B) ? TCLB_LAUNCH_PAIRS : 0) | (B->paths & TCLB_BATCH_SHORT_TILES);
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
  BCK(cudaMemcpyAsync(B->h_status, B->d_status, sizeof(int2) * B->cases.size(), cudaMemcpyDeviceToHost,
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
