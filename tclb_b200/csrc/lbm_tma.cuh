// Tile-staged iteration for 16-bit storage: a persistent kernel whose tiles
// (R whole rows of one z plane) are copied into shared memory by TMA through
// an S-stage mbarrier pipeline, then updated two nodes per thread.
//
// Why: with 16-bit densities the one-node and register-pair kernels are
// limited by issue slots and by how many loads their registers can keep in
// flight. Here the tensor-memory accelerator moves every population row of
// the next S-1 tiles while the threads compute the current one, so memory
// latency is hidden by the pipeline rather than by warps, and a pulled value
// is one shared-memory load.
//
// Layout of a stage: Q population blocks then one flag block, each R rows of
// nx 16-bit values (row-major, x fastest). For population i the block holds
// the rows the tile pulls from: source row (y - e_y) mod ny of plane
// (z - e_z) mod nz. A whole row is resident, so the x wrap is an index
// modulo nx. Rows that do not wrap come as one R-row box; at the y faces the
// rows come one by one (a second tensor map with a one-row box).
//
// Pipeline: a producer warp fills stage s (full[s] counts the bytes in);
// eight consumer warps wait on full[s], read their values, release the stage
// (one arrival each on empty[s]) and then compute, so copies of the next
// tiles overlap the arithmetic. No block-wide barrier after set-up.
//
// Failure: every wait on an mbarrier is bounded (about a second of clock).
// A warp whose wait runs out records an error code for the host and returns;
// the other warps' waits then run out in turn, so the kernel always ends.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "lbm_kernels.cuh"

namespace tclb {

struct TmaMaps {
  CUtensorMap rows;  // densities of the source snapshot: dims (nx, ny, nz, Q), box (nx, R, 1, 1)
  CUtensorMap row1;  // same tensor, box (nx, 1, 1, 1)
  CUtensorMap flags;  // node types: dims (nx, ny, nz), box (nx, R, 1)
};

// Tiles of the tile-staged kernels: 16-bit storage, nx a multiple of 32
// (TCLB pads nx so) up to 512. A row is one TMA box: up to 256 values as one
// box row (TMA boxes are at most 256 values along a dimension), wider rows as
// a (32, nx/32) box of a tensor whose x axis is split in two (32 x nx/32),
// which lands in shared memory in the same row-major order. In shared memory
// the rows of a tile lie `pitch` values apart: nx rounded up to a multiple of
// 64 for rows of at most 256 (the box is that wide; the values past nx are
// the copy's out-of-range zero fill), so that every row a TMA copy writes
// starts on a 128-byte boundary; rows wider than 256 come one per tile.
// R, the rows per tile, is the largest count with R * pitch <= 512 that
// divides ny; 0 where the kernel does not apply.
constexpr int TMA_MAX_NX = 512;
__host__ __device__ inline bool tma_wide(int nx) { return nx > 256; }
__host__ __device__ inline int tma_pitch(int nx) { return tma_wide(nx) ? nx : (nx + 63) / 64 * 64; }
inline int tma_rows_for(size_t elem, int nx, int ny) {
  if (elem != 2 || nx < 32 || nx % 32 || nx > TMA_MAX_NX) return 0;
  for (int R = 512 / tma_pitch(nx); R >= 1; R--)
    if (ny % R == 0) return R;
  return 0;
}
// Threads of a tile-staged block: the tile's node pairs, rounded up to whole
// warps, and one producer warp.
inline int tma_threads(int R, int nx) { return ((R * nx / 2 + 31) / 32 + 1) * 32; }  // R * nx / 2 pairs

// The driver's cuTensorMapEncodeTiled, reached through the runtime's
// entry-point query so the library links only the runtime; null if absent.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    EncodeTiledFn f = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
    return f;
  }();
  return fn;
}

// The three maps of one snapshot (16-bit values, planes `stride` apart) and
// its node types: rows (nx, ny, nz, Q) with an (nx, R, 1, 1) box, the same
// tensor with a one-row box, and the node types (nx, ny, nz) with an
// (nx, R, 1) box. False if the encoder is missing or refuses.
inline bool encode_tile_maps(void* buf, const void* flags, int nx, int ny, int nz, int Q, size_t stride, int R,
                             CUtensorMap* rows, CUtensorMap* row1, CUtensorMap* fmap) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t e = 2;
  if (tma_wide(nx)) {  // x split as (32, nx/32): rows (32, nx/32, ny, nz, Q), node types (32, nx/32, ny, nz)
    const cuuint32_t xo = (cuuint32_t)(nx / 32);
    const cuuint64_t dims[5] = {32, xo, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)Q};
    const cuuint64_t strides[4] = {32 * e, nx * e, (cuuint64_t)nx * ny * e, stride * e};
    const cuuint32_t box_rows[5] = {32, xo, (cuuint32_t)R, 1, 1};
    const cuuint32_t box_row1[5] = {32, xo, 1, 1, 1};
    const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
    if (enc(rows, CU_TENSOR_MAP_DATA_TYPE_UINT16, 5, buf, dims, strides, box_rows, ones,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    if (enc(row1, CU_TENSOR_MAP_DATA_TYPE_UINT16, 5, buf, dims, strides, box_row1, ones,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    const cuuint64_t fdims[4] = {32, xo, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t fstrides[3] = {32 * e, nx * e, (cuuint64_t)nx * ny * e};
    const cuuint32_t fbox[4] = {32, xo, (cuuint32_t)R, 1};
    return enc(fmap, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, const_cast<void*>(flags), fdims, fstrides, fbox, ones,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  const cuuint32_t pitch = (cuuint32_t)tma_pitch(nx);  // box width: nx rounded up to 64, zero-filled past nx
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)Q};
  const cuuint64_t strides[3] = {nx * e, (cuuint64_t)nx * ny * e, stride * e};
  const cuuint32_t box_rows[4] = {pitch, (cuuint32_t)R, 1, 1};
  const cuuint32_t box_row1[4] = {pitch, 1, 1, 1};
  const cuuint32_t ones[4] = {1, 1, 1, 1};
  if (enc(rows, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, buf, dims, strides, box_rows, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  if (enc(row1, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, buf, dims, strides, box_row1, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const cuuint64_t fdims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t fstrides[2] = {nx * e, (cuuint64_t)nx * ny * e};
  const cuuint32_t fbox[3] = {pitch, (cuuint32_t)R, 1};
  return enc(fmap, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, const_cast<void*>(flags), fdims, fstrides, fbox, ones,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Stages (shared memory per block: 128 + 3 * (Q+1) * 1 KB), two blocks per
// SM. Three suffice: for d3q19, whose tiles compute fastest, 4 and 5 stages
// measured the same.
template <class M>
constexpr int tma_stages() {
  return 3;
}
constexpr int TMA_CONSUMERS = 8;                   // consumer warps per block
constexpr unsigned TMA_TILE = TMA_CONSUMERS * 64;  // nodes per tile (two per consumer thread)

// Dynamic shared memory of the tile-staged kernels: 128 bytes of mbarriers,
// then the stages, laid out with the compile-time stride TMA_TILE per
// population block whatever the tile's R * nx (at most TMA_TILE; 384 when
// nx = 192), so the allocation must cover the full stride.
template <class M>
constexpr size_t tma_smem_bytes() {
  return 128 + (size_t)tma_stages<M>() * (M::Q + 1) * TMA_TILE * 2;
}
constexpr long long TMA_WAIT_CYCLES = 2000000000LL;  // ~1 s at 2 GHz
constexpr int TMA_ERR_TIMEOUT = 1;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity; false when it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, long long limit = TMA_WAIT_CYCLES) {
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// A producer leaving on a timeout first waits (bounded again) for the copies
// it issued into the other stages -- those of the tiles n-S+1 .. n-1, armed
// last -- so that none is still in flight into shared memory when the block
// exits. A stage whose copies were never issued just runs out once more.
__device__ __forceinline__ void tma_drain(unsigned long long* full, int S, int n, long long limit) {
  for (int j = n - S + 1 < 0 ? 0 : n - S + 1; j < n; j++)
    mbar_wait(static_cast<unsigned>(__cvta_generic_to_shared(&full[j % S])), (unsigned)(j / S) & 1u, limit);
}

__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_5d(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Issue the copies of the tile of rows y0 .. y0+R-1 of plane z into one
// stage; called by the whole producer warp after lane 0 has armed the stage's
// full barrier. Lane i < Q copies population i (one R-row box, or R one-row
// boxes where the rows wrap at a y face), lane Q the node types.
template <class M>
__device__ __forceinline__ void tma_fill_at(const CUtensorMap* rows, const CUtensorMap* row1,
                                            const CUtensorMap* flags, unsigned short* stage, unsigned bar, int z,
                                            int y0, int nx, int ny, int nz, int R, int lane) {
  constexpr unsigned block = TMA_TILE;  // values per population block (R * nx at most)
  const bool wide = tma_wide(nx);        // coordinates (0, 0, y, z, i) of the split-x maps
  if (lane < M::Q) {
    const int i = lane;
    const int ey = M::ey(i), ez = M::DIM == 2 ? 0 : M::ez(i);
    int zs = z - ez;
    zs = zs < 0 ? zs + nz : (zs >= nz ? zs - nz : zs);
    const unsigned dst = smem_u32(stage + (size_t)i * block);
    const int ys = y0 - ey;
    if (ys >= 0 && ys + R <= ny) {
      if (wide) tma_load_5d(dst, rows, 0, 0, ys, zs, i, bar);
      else tma_load_4d(dst, rows, 0, ys, zs, i, bar);
    } else {  // rows wrap at a y face: one row at a time
      for (int r = 0; r < R; r++) {
        int y = ys + r;
        y = y < 0 ? y + ny : (y >= ny ? y - ny : y);
        if (wide) tma_load_5d(dst + (unsigned)(r * nx * 2), row1, 0, 0, y, zs, i, bar);
        else tma_load_4d(dst + (unsigned)(r * tma_pitch(nx) * 2), row1, 0, y, zs, i, bar);
      }
    }
  } else if (lane == M::Q) {
    if (wide) tma_load_4d(smem_u32(stage + (size_t)M::Q * block), flags, 0, 0, y0, z, bar);
    else tma_load_3d(smem_u32(stage + (size_t)M::Q * block), flags, 0, y0, z, bar);
  }
}

// Tile t of a lattice (tiles of R rows, z-major).
template <class M>
__device__ __forceinline__ void tma_fill(const TmaMaps& T, unsigned short* stage, unsigned bar, int t, int nx,
                                         int ny, int nz, int R, int lane) {
  const int rows_per_plane = ny / R;
  const int z = t / rows_per_plane, y0 = (t % rows_per_plane) * R;
  tma_fill_at<M>(&T.rows, &T.row1, &T.flags, stage, bar, z, y0, nx, ny, nz, R, lane);
}

// The kernel: ncons = ceil(R*nx/64) <= TMA_CONSUMERS warps update node
// pairs (threads past the tile's R*nx/2 pairs only take part in the stage
// protocol), one more warp (the last) produces. Block = (ncons + 1) * 32 threads; the
// consumer warps cover the tile's R*nx/2 pairs, one pair per thread. Grid = resident blocks
// (persistent), walking tiles t = blockIdx.x + k*gridDim.x.
// Dynamic shared memory: 128 bytes of mbarriers (full[S], empty[S]), then
// TMA_STAGES stages.
constexpr int TMA_THREADS = (TMA_CONSUMERS + 1) * 32;

// FAULT (the failure-path test, set only by tclb_set_fault_injection):
// wait_cycles bounds every mbarrier wait instead of the fixed bound, and the
// producer arms tile skip_tile's stage but issues none of its copies, so its
// consumers' wait runs out. Without FAULT both parameters are ignored and
// the waits keep the compile-time bound.
// PARTIAL: the tile's pairs do not fill whole warps (R * nx / 2 not a
// multiple of 32), so consumer threads check that they hold a pair.
template <class M, class R, class St, bool FAULT = false, bool PARTIAL = false, bool LANES = false>
__global__ void __launch_bounds__(TMA_THREADS, 2)
    k_iterate_tma(const Args<R, M::NSET> a, const __grid_constant__ TmaMaps T,
                  const PlaneAddr<typename St::T, M::Q> P, int R_rows, int* err, long long wait_cycles_arg,
                  int skip_tile) {
  const long long wait_cycles = FAULT ? wait_cycles_arg : TMA_WAIT_CYCLES;
  static_assert(M::Q < 32, "one producer lane per population plus one for the node types");
  using P16 = Pack16<St>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);
  constexpr int TMA_STAGES = tma_stages<M>();
  static_assert(TMA_STAGES <= 8, "128 bytes hold 8 full and 8 empty barriers");
  unsigned long long* empty = full + 8;
  unsigned short* stages = reinterpret_cast<unsigned short*>(smem + 128);
  const int nx = a.nx, ny = a.ny, nz = a.nz, pitch = tma_pitch(nx);
  constexpr unsigned block = TMA_TILE;  // R_rows * pitch at most: a compile-time stride for the stage layout
  constexpr unsigned stage_elems = (M::Q + 1) * block;
  const int ntiles = nz * (ny / R_rows);
  const int rows_per_plane = ny / R_rows;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncons = (int)(blockDim.x >> 5) - 1;

  if (tid == 0) {
    for (int s = 0; s < TMA_STAGES; s++) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), ncons);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();  // the only block-wide barrier

  if (warp == ncons) {  // producer
    for (int k = 0;; k++) {
      const int t = blockIdx.x + k * gridDim.x;
      if (t >= ntiles) break;
      const int s = k % TMA_STAGES;
      const unsigned fb = smem_u32(&full[s]);
      bool ok = true;
      if (lane == 0 && k >= TMA_STAGES)
        ok = mbar_wait(smem_u32(&empty[s]), (unsigned)(k / TMA_STAGES - 1) & 1u, wait_cycles);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          atomicExch(err, TMA_ERR_TIMEOUT);
          tma_drain(full, TMA_STAGES, k, wait_cycles);
        }
        return;
      }
      if (lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(fb, (unsigned)(M::Q + 1) * (unsigned)(R_rows * pitch) * 2u);  // R_rows boxed rows
      }
      __syncwarp();
      if (!FAULT || t != skip_tile) tma_fill<M>(T, stages + s * stage_elems, fb, t, nx, ny, nz, R_rows, lane);
    }
    return;
  }

  // consumers
  const int half = nx >> 1;
  const int r = tid / half, x = 2 * (tid % half);  // a warp may span two rows (nx a multiple of 32)
  const bool act = !PARTIAL || r < R_rows;         // threads past the tile's pairs

  const int xm = x == 0 ? nx - 1 : x - 1, xp2 = x + 2 == nx ? 0 : x + 2;
  // tile t = (z, yt) with yt = t mod rows_per_plane, stepped by gridDim.x per
  // round without a division; the stage index and its phase likewise
  const int dz = (int)gridDim.x / rows_per_plane, dyt = (int)gridDim.x % rows_per_plane;
  int z = (int)blockIdx.x / rows_per_plane, yt = (int)blockIdx.x % rows_per_plane;
  int s = 0;
  unsigned phase = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const bool ok = mbar_wait(smem_u32(&full[s]), phase, wait_cycles);
    if (!__all_sync(0xffffffffu, ok)) {  // the warp leaves together
      if (lane == 0) atomicExch(err, TMA_ERR_TIMEOUT);
      return;
    }
    const unsigned short* st = stages + s * stage_elems;
    const unsigned short* mine = st + r * pitch;  // this thread's row in population block 0
    const int y = yt * R_rows + r;
    float2 v[M::Q];
    unsigned fl2 = 0;
    if (act) {
#pragma unroll
      for (int i = 0; i < M::Q; i++) {
        const unsigned short* row = mine + i * block;  // constant offset per population
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
    const unsigned node = (unsigned)x + (unsigned)nx * ((unsigned)y + (unsigned)ny * (unsigned)z);
    if (++s == TMA_STAGES) {
      s = 0;
      phase ^= 1u;
    }
    z += dz;
    yt += dyt;
    if (yt >= rows_per_plane) {
      yt -= rows_per_plane;
      z++;
    }
    if (act)
      pair_update_store<M, R, St, PlaneAddr<typename St::T, M::Q>, Args<R, M::NSET>, LANES>(
          v, (flag_t)(fl2 & 0xffffu), (flag_t)(fl2 >> 16), a, P, node);
  }
}

}  // namespace tclb
