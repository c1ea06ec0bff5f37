/*
 * tclb_b200 -- C ABI of the B200 lattice-Boltzmann engine.
 *
 * Drop-in for the Run path of TCLB's `Lattice` class (src/Lattice.h.Rt:39-191)
 * for the d2q9, d3q19 and d3q27_cumulant models. Every entry point returns a
 * status (TCLB_OK = 0, negative on error) instead of exiting the process as
 * TCLB's HANDLE_ERROR does (src/cross.cu:24-32); tclb_last_error() gives the
 * message. Handles are independent, so many lattices may live in one process
 * and on one GPU (TCLB keeps one lattice per process in __constant__ memory).
 *
 * Buffers passed in are host memory owned by the caller unless stated
 * otherwise; pinned host memory makes the copies asynchronous-capable.
 * `stream` arguments are cudaStream_t values passed as void* (NULL = the
 * lattice's own stream).
 */
#ifndef TCLB_B200_H
#define TCLB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tclb_lattice* tclb_h;

/* models */
#define TCLB_MODEL_D2Q9 0
#define TCLB_MODEL_D3Q19 1
#define TCLB_MODEL_D3Q27_CUMULANT 2

/* arithmetic precision of the collision (real_t) */
#define TCLB_FP32 0
#define TCLB_FP64 1

/* storage format of the densities (storage_t); *_SHIFT stores f_i - w_i */
#define TCLB_STORAGE_SAME 0
#define TCLB_STORAGE_FP16 1
#define TCLB_STORAGE_FP16_SHIFT 2
#define TCLB_STORAGE_BF16 3
#define TCLB_STORAGE_BF16_SHIFT 4

/* iteration flags, same values as src/Lattice.h.Rt:19-31 */
#define TCLB_ITER_NORM 0x001
#define TCLB_ITER_GLOBS 0x010
#define TCLB_ITER_INTEG 0x070
#define TCLB_ITER_LASTGLOB 0x080

#define TCLB_OK 0
#define TCLB_ERR_ARG (-1)
#define TCLB_ERR_CUDA (-2)
#define TCLB_ERR_MEMORY (-3)
#define TCLB_ERR_STATE (-4)

/* Message of the last failing call on this thread. */
const char* tclb_last_error(void);

/* Model description: number of densities Q, Settings, ZoneSettings, Globals,
   Quantities, and the ZONE_SHIFT of the node-type word. Replaces the
   R-generated constants of src/conf.R:859-891. */
int tclb_model_info(int model, int* Q, int* nsettings, int* nzonesettings, int* nglobals, int* nquantities,
                    int* zone_shift);
/* Name of item `i` of kind 0 Setting, 1 ZoneSetting, 2 Global, 3 NodeType,
   4 Quantity; for NodeType also its value and group mask. */
int tclb_model_item(int model, int kind, int i, const char** name, int* value, int* mask);

/* Lattice(lbRegion, MPIInfo, nSnaps) (src/Lattice.cu.Rt:87-151): allocate the
   two snapshots, node types, zonal settings and Globals in one pooled device
   allocation on the current device. nx is used as given (TCLB's Solver pads
   it to a multiple of 32 before, src/Solver.cpp.Rt:273). Settings start at
   their defaults (src/Solver.cpp.Rt:276-281, :393). */
int tclb_create(tclb_h* out, int model, int nx, int ny, int nz, int precision, int storage);
int tclb_destroy(tclb_h h);
int tclb_get_size(tclb_h h, int* nx, int* ny, int* nz);

/* Lattice::FlagOverwrite (src/Lattice.cu.Rt:1040-1054): copy a box of node
   types (TCLB bit layout, x fastest) at offset (dx,dy,dz). */
int tclb_set_flags(tclb_h h, const uint16_t* flags, int dx, int dy, int dz, int nx, int ny, int nz);
int tclb_get_flags(tclb_h h, uint16_t* flags);

/* Lattice::SetSetting (src/Lattice.cu.Rt:1350-1358): set and follow the
   derived-setting chain (e.g. d2q9 Viscosity -> RelaxationRate -> S2). */
int tclb_set_setting(tclb_h h, int setting, double value);
int tclb_get_setting(tclb_h h, int setting, double* value);
/* ZoneSettings::set (src/ZoneSettings.h:58-77); zone = -1 sets every zone. */
int tclb_set_zone_setting(tclb_h h, int zone_setting, int zone, double value);
/* ZoneSettings::get (src/ZoneSettings.h) for one zone. */
int tclb_get_zone_setting(tclb_h h, int zone_setting, int zone, double* value);

/* Lattice::Init (src/Lattice.cu.Rt:799-821): BaseInit stage (equilibrium
   from settings), resets the iteration counter and the Globals. */
int tclb_init(tclb_h h);

/* Every node set to the model's equilibrium (SetEquilibrum of each model's
   Dynamics.c.Rt) at density rho[n] and momentum rho[n]*u[3n..3n+2]; arrays
   are real_t (float for TCLB_FP32, double for TCLB_FP64), x fastest. This is
   the initial condition that TCLB can only inject through <LoadBinary>
   (src/Handlers/acLoadBinary.cpp:5-23). Resets the iteration counter and the
   Globals like tclb_init. */
int tclb_init_equilibrium(tclb_h h, const void* rho, const void* u, void* stream);

/* Lattice::Iterate (src/Lattice.cu.Rt:900-989) for ITER_NORM: `niter`
   pull-stream+collide iterations. ITER_LASTGLOB integrates Globals on the last
   iteration only and replaces the host Globals with them; ITER_INTEG
   integrates on every iteration and adds them. */
int tclb_iterate(tclb_h h, int niter, int iter_type, void* stream);

/* Lattice::globals[] after calcGlobals (src/Lattice.cu.Rt:1279-1315), FP64, in
   TCLB order: SUM globals, Objective, MAX globals. */
int tclb_get_globals(tclb_h h, double* out);
int tclb_clear_globals(tclb_h h);

/* Lattice::GetQuantity (src/Lattice.cu.Rt:1184-1222): quantity `q` over the
   region (x0,y0,z0,nx,ny,nz) times `scale`, in the lattice's real_t (float for
   TCLB_FP32, double for TCLB_FP64); vector quantities are 3 values per node. */
int tclb_get_quantity(tclb_h h, int q, const int region[6], void* out, double scale, void* stream);

/* Lattice::Color (src/Lattice.cu.Rt:791-793 -> LatticeContainer::Color,
   src/LatticeContainer.inc.cpp.Rt:350-423), headless: nx*ny RGBA bytes (uchar4,
   x fastest) of plane z (z < 0: nz/2, the plane TCLB draws) from the model's
   Color() through TCLB's colour map. `rgba` is device memory, written
   asynchronously on `stream`, or host memory when on_host != 0 (the call then
   returns after the copy). */
int tclb_color(tclb_h h, void* rgba, int z, int on_host, void* stream);

/* Flow diagnostics of the current snapshot (no TCLB counterpart: TCLB has no
   such Globals, its users reduce an exported U field): out[0] = kinetic energy
   1/2 sum |U|^2, out[1] = enstrophy 1/2 sum |curl U|^2, in lattice units, with
   U the model's velocity quantity and the curl by second-order central
   differences on the periodic lattice; FP64 sums over all nodes. Uses the
   quantity staging buffer (allocated on first use); returns after the copy. */
int tclb_energy_enstrophy(tclb_h h, double* out, void* stream);

/* Same result as tclb_get_quantity, for callers that must not allocate device
   memory: an application whose GPU memory is all owned by its own pool or
   admission budget, or a latency-critical loop where cudaMalloc/cudaFree would
   synchronise the device. No counterpart in the reference (TCLB's GetQuantity
   allocates a buffer on every call, src/Lattice.cu.Rt:1210-1220).
   It stages the quantity in a fixed 8 MiB device array compiled into the
   library (held by every GPU that loads the library until the process exits)
   and calls no cudaMalloc/cudaFree. Regions whose quantity needs more than
   8 MiB (nodes x components x sizeof(real_t)) are rejected with
   TCLB_ERR_ARG. The call ends by synchronising its stream, so it cannot be
   captured into a CUDA graph. The first call on each device looks up the
   array's device address (cudaGetSymbolAddress) and caches it; make that
   first call before another thread of the process starts a global-mode
   stream capture. All calls share the array: calls that overlap on the GPU
   race. */
int tclb_get_quantity_noalloc(tclb_h h, int q, const int region[6], void* out, double scale, void* stream);

/* Get_/Set_<field> for all densities at once: SoA [q][z][y][x] as double. */
int tclb_get_densities(tclb_h h, double* out);
int tclb_set_densities(tclb_h h, const double* in);

/* Raw snapshot of the current densities in storage format (Lattice::save /
   load, src/Lattice.cu.Rt:642-769, without TCLB's margin split). */
size_t tclb_snapshot_bytes(tclb_h h);
int tclb_save(tclb_h h, void* host, size_t bytes, void* stream);
int tclb_load(tclb_h h, const void* host, size_t bytes, void* stream);

/* TCLB's .pri checkpoint of the current snapshot (Lattice::save / load,
   src/Lattice.cu.Rt:642-769): the snapshot's non-empty margin blocks in block
   order, each an x-fastest box of storage_t values per density, byte for byte
   what a single-rank TCLB run of the same model and storage writes: an edge
   node's outgoing density sits in the margin block it is pulled from (and, for
   d3q27_cumulant only, in place as well); slots TCLB never writes are zero.
   Loading takes each node's value from the block it is pulled from. */
size_t tclb_pri_bytes(tclb_h h);
int tclb_save_pri(tclb_h h, void* host, size_t bytes);
int tclb_load_pri(tclb_h h, const void* host, size_t bytes);

/* Iterations done since Init, and the bytes one iteration moves
   (2*Q*sizeof(storage_t) + sizeof(flag_t) per node). */
int tclb_get_iteration(tclb_h h, long long* iter);
double tclb_bytes_per_update(tclb_h h);

/* Synchronise the lattice's stream. */
int tclb_sync(tclb_h h);

/* Launch shape of the iteration kernel (bx multiple of 32, bx*by <= 256) and
   flags: TCLB_LAUNCH_GRAPHS replays runs of plain iterations from a captured
   CUDA graph (on by default); TCLB_LAUNCH_PAIRS lets 16-bit storage with
   nx % 64 == 0 update two nodes per thread on plain iterations: 32-bit
   accesses, and for d3q19 / d3q27_cumulant bulk nodes one packed FP32x2
   collision for both (on by default); TCLB_LAUNCH_TMA lets 16-bit storage
   stage tiles of whole rows in shared memory with TMA on plain iterations
   (on by default; it takes precedence over PAIRS) when nx is a multiple of 32
   up to 512 (tiles of whole rows, at most 512 nodes, the number of rows
   dividing ny). bx, by shape the one-node kernel.
   A staging wait that runs out (about a second) is reported as TCLB_ERR_CUDA
   by the next tclb_sync or Globals-reading tclb_iterate. */
#define TCLB_LAUNCH_GRAPHS 1
#define TCLB_LAUNCH_PAIRS 2
#define TCLB_LAUNCH_TMA 4
/* With TCLB_LAUNCH_TMA: stage tiles wherever the tile-staged kernel applies,
   also where d3q19 otherwise takes the register pair kernel (nx % 64 == 0 and
   rows wider than 256, tiles of fewer than 448 nodes, or fewer than four tiles
   per resident block: measured faster there). */
#define TCLB_LAUNCH_TMA_ALWAYS 8
int tclb_set_launch(tclb_h h, int bx, int by, int flags);
/* The launch shape and the paths plain iterations take on this lattice: the
   flags that are both enabled and applicable (no TCLB counterpart). */
int tclb_get_launch(tclb_h h, int* bx, int* by, int* flags);
/* Failure-path test of the tile-staged kernel (no TCLB counterpart; TCLB
   exits on a CUDA error, src/cross.cu:24-32): plain iterations run with
   every staging wait bounded by wait_cycles SM clock cycles (0: the default,
   about a second) and, when tile >= 0, the producer arms that tile's stage
   without issuing its copies, so the wait of its consumers runs out. The
   iteration then leaves that tile's nodes unwritten, and the next tclb_sync
   returns TCLB_ERR_CUDA, reports it in tclb_last_error() and clears the
   device error word. tile = -1 and wait_cycles = 0 restore normal runs.
   Nothing faults: the kernel returns after its bounded waits. */
int tclb_set_fault_injection(tclb_h h, int tile, long long wait_cycles);

/* ---------------------------------------------------------------------------
   XML case files (<CLBConfig>): the control flow of TCLB's main and handler
   tree for the Run path (src/main.cpp:173-425, src/Handlers/acGeometry.cpp,
   acModel.cpp, acParam.cpp, acInit.cpp, acSolve.cpp, acContainer.cpp,
   acRepeat.cpp, cbLog.cpp, cbBIN.cpp, cbFailcheck.cpp, cbStop.cpp, cbVTK.cpp,
   cbTXT.cpp, cbSaveBinary.cpp, cbSample.cpp, cbPID.cpp, cbKeep.cpp,
   cbAveraging.cpp, IfContainer.cpp). Values may carry units ("1e-6m2/s",
   "5mm+1cm");
   <Units><Param value= gauge=> elements fix the lattice scale of each base
   unit as src/unit.cpp does, and the Log's _si columns use those scales.
   Unknown unit symbols are errors here (TCLB reads them as 0).
   ------------------------------------------------------------------------- */
const char* tclb_case_last_error(void);
/* Node types of a case's <Geometry>, rasterised like src/Geometry.cpp.Rt with
   nx padded to a multiple of 32 (src/Solver.cpp.Rt:273). dims gets nx, ny, nz;
   pass flags = NULL to query the size first. */
int tclb_case_geometry(const char* xml_text, int model, int dims[3], uint16_t* flags, size_t capacity);
/* Run a case file for one model. Output files are named like
   Solver::outIterFile (src/Solver.h.Rt:102-105): <out_dir><case>_<Log|BIN>_P00_<iteration>... */
int tclb_case_run(const char* xml_path, int model, int precision, int storage, const char* out_dir, int verbose);

/* ---------------------------------------------------------------------------
   Batches: many independent cases of one model advanced together by one
   persistent, CUDA-graph-captured launch per replay. No counterpart in the
   reference, which runs one lattice per process (src/main.cpp:173-425).
   ------------------------------------------------------------------------- */
typedef struct tclb_batch* tclb_batch_h;

const char* tclb_batch_last_error(void);

/* Device bytes one case occupies (two snapshots, node types, zonal table,
   Globals, and tensor maps where the tile-staged kernel applies): the
   footprint that admission compares with the budget. */
size_t tclb_batch_case_bytes(int model, int precision, int storage, int nx, int ny, int nz);

/* A batch admits cases while the sum of their footprints stays within
   budget_bytes and at most max_cases are resident. */
int tclb_batch_create(tclb_batch_h* out, int model, int precision, int storage, size_t budget_bytes, int max_cases);
int tclb_batch_destroy(tclb_batch_h b);
/* Grow the batch's device memory pool to hold at least `bytes` (at most the
   budget) for the cases it will admit: blocks of up to 2 GiB are allocated
   and freed back to the pool, which keeps freed memory. Admissions that fit
   the reserve then take memory from the pool without mapping new device
   memory, which otherwise costs milliseconds per case, and at times hundreds
   of milliseconds, while other work runs. Returns after the pool has grown;
   TCLB_ERR_MEMORY if the device cannot provide it (the pool keeps what it
   got). The reserve does not count against the budget. No TCLB counterpart. */
int tclb_batch_reserve(tclb_batch_h b, size_t bytes);

/* Admit a case: node types (x fastest), the full Settings vector (derived
   chains already applied), `zone_rows` rows of ZoneSettings (zone 0..), and
   the number of iterations to run. The case starts at its BaseInit
   equilibrium. TCLB_ERR_MEMORY when the budget or the slots are exhausted. */
int tclb_batch_add_case(tclb_batch_h b, int nx, int ny, int nz, const uint16_t* flags, const double* settings,
                        const double* zone_settings, int zone_rows, int niter, int* case_id);
/* Retire a case and return its memory to the batch's pool (stream-ordered). */
int tclb_batch_remove_case(tclb_batch_h b, int case_id);

/* Launch shape: tiles of bx x by nodes (bx a multiple of 32 up to 256, by up
   to 256), iterations per replay, and grid: 0 (default) = one block per tile,
   > 0 = a persistent grid of that many blocks walking the tiles, < 0 =
   persistent with SMs x resident blocks. A block has bx x min(by, 256 / bx)
   threads and walks the tile's rows. One block per tile measured fastest on
   mixed sizes. */
int tclb_batch_set_launch(tclb_batch_h b, int bx, int by, int iters_per_launch, int grid_blocks);
/* Run the batch's work on a high-priority stream (high != 0) or a normal one:
   with batches of different models running at once, the blocks of the
   high-priority batch are scheduled first (e.g. small cases that should not
   wait behind large ones). Waits for the batch's work in flight. */
int tclb_batch_set_priority(tclb_batch_h b, int high);
int tclb_batch_get_launch(tclb_batch_h b, int* bx, int* by, int* iters_per_launch);
/* Paths of the plain launches: TCLB_LAUNCH_PAIRS (on by default) lets 16-bit
   storage update two neighbouring nodes per thread with 32-bit accesses when
   the tile width bx is a multiple of 64 and the grid is one block per tile
   (blocks of bx / 2 x min(by, T / (bx / 2)) threads, T = 256, 128 for
   d3q27_cumulant); the Globals launch keeps the one-node kernel.
   TCLB_LAUNCH_TMA (on by default) runs the plain launches of each 16-bit case
   whose rows fit the tile-staged kernel (nx a multiple of 32 up to 512) through
   it, tensor maps kept with the case;
   the other cases take the pair or one-node form. A staging wait that runs
   out (about a second) is reported as TCLB_ERR_CUDA by the next
   tclb_batch_sync. TCLB_BATCH_ADAPTIVE (on by default) fits the launches to
   the live work: it halves the tile height, down to the block's thread rows,
   while the live cases would give fewer tiles than two waves of resident
   blocks, and leaves the tile-staged kernel out while the staged cases give
   fewer than 8 tiles per resident block (its pipeline start would dominate);
   off, tiles are always by rows high and every case that fits is staged.
   TCLB_BATCH_GLOBALS_AT_END (off by default) computes a case's Globals only
   in the replay where it finishes (tclb_batch_get_globals then holds the
   Globals of its last iteration once it is done, zeros before): the last
   launch of the other replays runs the faster plain kernels for it.
   get_paths gives the flags that are enabled and apply to the current launch
   shape (TCLB_LAUNCH_TMA: to at least one live case). No TCLB counterpart. */
#define TCLB_BATCH_ADAPTIVE 8
#define TCLB_BATCH_GLOBALS_AT_END 16
int tclb_batch_set_paths(tclb_batch_h b, int flags);
int tclb_batch_get_paths(tclb_batch_h b, int* flags);

/* Enqueue one replay (asynchronous); every active case advances by
   min(iters_per_launch, remaining) iterations; Globals are those of each case's
   last iteration in the replay. */
int tclb_batch_step(tclb_batch_h b);
int tclb_batch_sync(tclb_batch_h b);
/* 1 when the batch's enqueued work has finished (tclb_batch_sync then returns
   at once), 0 while it runs, negative on error; never blocks. */
int tclb_batch_done(tclb_batch_h b);
/* After tclb_batch_sync: iterations done / left for a case. */
int tclb_batch_poll(tclb_batch_h b, int case_id, long long* iterations_done, int* remaining);
int tclb_batch_get_globals(tclb_batch_h b, int case_id, double* out);
int tclb_batch_get_quantity(tclb_batch_h b, int case_id, int q, void* out, double scale);
int tclb_batch_info(tclb_batch_h b, int* ncases_active, int* ntiles, size_t* used_bytes, size_t* budget_bytes);
/* Node updates the next step will perform (as of the last status read-back). */
long long tclb_batch_pending_updates(tclb_batch_h b);

#ifdef __cplusplus
}
#endif
#endif
