/*
 * zsph.h -- C ABI of the B200-native delta-SPH single-GPU step.
 *
 * The entry points replace the reference solver's single-GPU hot path
 * (ZSPH, single_gpu_sph_src/) for a caller that drives it the way
 * single_gpu_sph_src/deltasph/main.cu does.  All structs are plain C; every
 * device pointer is caller-owned; every call returns a ZSPH_* status and
 * never exits the process.  The float arrays of a particle buffer must start
 * on an 8-byte boundary (as cudaMalloc and zsph_alloc_ptc give them); calls
 * given others return ZSPH_EINVAL (ZSPH_ECUDA from the learned and
 * precision-form entry points) without launching anything.  `stream` is a cudaStream_t passed as void*
 * (NULL = the legacy default stream).
 *
 * Particle layout (unchanged from the reference, data_structure.cuh:158-182):
 * pos, vel, tmp_pos, tmp_vel hold 3 floats per particle (float3), rhop and
 * tmp_rhop 2 floats (float2: density, pressure), acc_drhodt and
 * dofv_grandrho 4 floats (float4), type/table/index/hash one int, and
 * grid_start/grid_end one int per grid cell.  Particle type 1 is fluid,
 * any other type a dummy wall, 100 a particle that left the grid.
 */
#ifndef ZSPH_H
#define ZSPH_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ZSPH_OK = 0,
  ZSPH_EINVAL = 1,   /* bad argument, dt > dt_max, size mismatch, unsupported grid factor */
  ZSPH_ECUDA = 2,    /* a CUDA runtime call failed; see zsph_last_error */
  ZSPH_ENAN = 3,     /* a non-finite acceleration or density was produced */
  ZSPH_ETIMEOUT = 4, /* a bounded device-side wait gave up */
  ZSPH_EIO = 5,      /* file or JSON error */
  ZSPH_ENOMEM = 6    /* device allocation failed */
};

/* Equation sets (zsph_set_equations): the reference builds deltasph with
 * -DZSPH_DELTA (equation/delta_ns.cu) and simplesph with -DZSPH_SIMPLE
 * (equation/simple_ns.cu) from the same sources. */
enum { ZSPH_EQ_DELTA = 0, ZSPH_EQ_SIMPLE = 1 };

/* Bits of the device status word (zsph_status). */
enum {
  ZSPH_FLAG_NAN = 1,         /* non-finite acc_drhodt or density */
  ZSPH_FLAG_KILLED = 2,      /* a particle left the grid and became type 100 */
  ZSPH_FLAG_NB_OVERFLOW = 4, /* a neighbour list overflowed (handled, slower path) */
  ZSPH_FLAG_BAD_KEY = 8,     /* zsph_sort_index got a hash outside [0, grid_num) */
  ZSPH_FLAG_TIMEOUT = 16     /* a bounded device-side wait gave up: a staging copy (slower path taken), the
                                search's scan look-back, or a persistent kernel's grid barrier */
};

/* cpu_json_t (single_gpu_sph_src/header/data_structure.cuh:6-51); the three
 * std::string members become fixed char arrays. */
typedef struct {
  float g, m, rho0, dx, h_factor, r_factor, eta_factor, cs_factor, delta, alpha;
  float xmin, xmax, ymin, ymax, zmin, zmax, grid_layer_factor, grid_size_factor;
  float dt;
  int start_step, current_step, end_step, output_step;
  int ptc_num, water_ptc_num, air_ptc_num, wall_ptc_num, rigid_ptc_num;
  int thread_num, gpu_id;
  char input_path[256], output_path[256], git_hash[64];
} zsph_json_t;

/* cpu_param_t (data_structure.cuh:53-105), same fields and order. */
typedef struct {
  float g, m, rho0, dx, h, r, eta, cs, adh, delta, alpha;
  float dt;
  int start_step, current_step, end_step, output_step;
  float xmin, xmax, ymin, ymax, zmin, zmax;
  int grid_factor;
  float grid_size;
  float grid_xmin, grid_ymin, grid_zmin, grid_xmax, grid_ymax, grid_zmax;
  int grid_xdim, grid_ydim, grid_zdim, grid_num, grid_hash_min, grid_hash_max;
  int ptc_num, water_ptc_num, air_ptc_num, wall_ptc_num, rigid_ptc_num;
  int thread_num, gpu_id;
  char input_path[256], output_path[256], git_hash[64];
} zsph_cpu_param_t;

/* gpu_param_t (data_structure.cuh:107-134), field for field. */
typedef struct {
  float half_dt, h, g, m, rho0, adh, h2, eta2, cs2, alpha, delta_h_cs, h_cs_rho_m;
  float grid_size;
  int grid_factor;
  float grid_xmin, grid_ymin, grid_zmin;
  int grid_xdim, grid_ydim, grid_zdim, grid_hash_min, grid_hash_max;
  int ptc_num;
} zsph_gpu_param_t;

/* gpu_ptc_t (data_structure.cuh:158-168): same layout (all members are pointers). */
typedef struct {
  float *pos, *vel, *rhop, *tmp_pos, *tmp_vel, *tmp_rhop;
  int *type, *table;
} zsph_ptc_t;

/* gpu_tmp_t (data_structure.cuh:170-182): same layout. */
typedef struct {
  float *acc_drhodt, *dofv_grandrho, *dofv;
  int *index, *hash, *grid_start, *grid_end;
} zsph_tmp_t;

typedef struct zsph_handle zsph_handle_t;

/* ---- host-side case set-up -------------------------------------------- */

/* read_json (single_gpu_sph_src/io/read_json.cu:5-51): reads the 33
 * required keys; a missing or mistyped key is ZSPH_EIO with its name in err. */
int zsph_read_json(const char* path, zsph_json_t* out, char* err, int errlen);
/* Optional keys of the same case file, which the reference's read_json
 * ignores (no counterpart in the reference; all may be absent):
 *   "equations": "delta" (default) or "simple": the equation set, which the
 *       reference picks when it is built (ZSPH_DELTA / ZSPH_SIMPLE,
 *       deltasph/CMakeLists.txt:25-31);
 *   "eos": "linear" (default): the equation of state of the reference's code,
 *       p = c0^2 (rho - rho0) (lib/time_int.cu:39-40); any other value is
 *       ZSPH_EINVAL, since no other one is implemented;
 *   "snapshot_every": k >= 0: zsph_compat_run writes a snapshot of the state
 *       after every k-th step as output_path/snapshot<s>.zsnap, s being the
 *       number of the next step to run (0: none);
 *   "resume": the path of such a snapshot: zsph_compat_run loads it after
 *       the input and continues from its step.
 * A mistyped or out-of-range value is ZSPH_EINVAL with its key in err. */
typedef struct {
  int equations;      /* ZSPH_EQ_DELTA or ZSPH_EQ_SIMPLE */
  int snapshot_every; /* 0: no snapshots */
  char resume[256];   /* empty: start from the input */
} zsph_case_options_t;
int zsph_read_case_options(const char* path, zsph_case_options_t* out, char* err, int errlen);

/* set_cpu_param (single_gpu_sph_src/lib/init.cu:153-219), including the
 * check_dt call of init.cu:218: returns ZSPH_EINVAL when dt > dt_max
 * (the reference exits, check.cu:9-17). */
int zsph_set_cpu_param(zsph_cpu_param_t* param, const zsph_json_t* jdata);

/* set_gpu_param (single_gpu_sph_src/lib/init.cu:221-251). */
int zsph_set_gpu_param(zsph_gpu_param_t* gparam, const zsph_cpu_param_t* cparam);

/* check_dt (single_gpu_sph_src/lib/check.cu:3-18): ZSPH_OK when
 * dt <= 0.25*h/sqrt(-g*(zmax-zmin)), else ZSPH_EINVAL; dt_max may be NULL. */
int zsph_check_dt(const zsph_cpu_param_t* param, float* dt_max);

/* ---- device buffers ----------------------------------------------------- */

/* alloc_gpu_ptc_data / delete_gpu_ptc_data (lib/init.cu:38-80). */
int zsph_alloc_ptc(zsph_ptc_t* ptc, int ptc_num);
int zsph_free_ptc(zsph_ptc_t* ptc);
/* alloc_gpu_tmp_data / delete_gpu_tmp_data (lib/init.cu:82-134); zero-filled. */
int zsph_alloc_tmp(zsph_tmp_t* tmp, int ptc_num, int grid_num);
int zsph_free_tmp(zsph_tmp_t* tmp);
/* cpu_to_gpu (lib/init.cu:136-151): host pos/vel/rhop/type/table/acc_drhodt
 * (acc_drhodt may be NULL: zero-filled) into the device buffers. */
int zsph_cpu_to_gpu(const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, const float* pos, const float* vel,
                    const float* rhop, const int* type, const int* table, const float* acc_drhodt,
                    int ptc_num, void* stream);
/* gpu_to_cpu (lib/gmemcpy.cu:3-36): device buffers to host arrays; any
 * NULL host pointer is skipped. */
int zsph_gpu_to_cpu(const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, float* pos, float* vel, float* rhop,
                    int* type, int* table, float* acc_drhodt, int* hash, int ptc_num, void* stream);

/* ---- solver handle -------------------------------------------------------- */

/* Creates a solver for one case.  Owns only its scratch (counting-sort
 * buckets, packed particle shadows, neighbour lists); allocates it here and
 * never during a step.  grid_num = grid_xdim*grid_ydim*grid_zdim
 * (cpu_param_t::grid_num).  Binds to the current CUDA device. */
int zsph_create(const zsph_gpu_param_t* gparam, int grid_num, zsph_handle_t** out);
void zsph_destroy(zsph_handle_t* h);
/* Replaces the constants (dt and physics) of an existing handle; the grid
 * and particle count must not change. */
int zsph_set_params(zsph_handle_t* h, const zsph_gpu_param_t* gparam);

/* Selects the equations of zsph_boundary, zsph_governing, zsph_step and
 * zsph_run: ZSPH_EQ_DELTA (default; equation/delta_ns.cu) or ZSPH_EQ_SIMPLE
 * (equation/simple_ns.cu, whose div(v) is the scalar tmp->dofv). */
int zsph_set_equations(zsph_handle_t* h, int equations);

/* cuda_ptc_hash (single_gpu_sph_src/lib/hash.cu:3-26): cell hash of every
 * particle into tmp->hash, identity into tmp->index, out-of-grid particles
 * become type 100 at the grid origin. */
int zsph_hash(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream);
/* cuda_sort_index (single_gpu_sph_src/lib/sort.cu:3-6): stable ascending
 * sort of tmp->hash carrying tmp->index.  Keys must lie in [0, grid_num). */
int zsph_sort_index(zsph_handle_t* h, const zsph_tmp_t* tmp, void* stream);
/* No counterpart in the reference.  The same stable sort as zsph_sort_index
 * for callers that cannot allocate device memory: it needs no handle (whose
 * creation calls cudaMalloc) and calls no allocator.  Its scratch is a fixed
 * static device array of about 3.2 MB, held by every GPU that loads the
 * library until the process exits, so it accepts at most 131072 particles
 * (gparam->ptc_num) and 131072 cells (grid_num) and returns ZSPH_EINVAL
 * beyond that.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress); make that call before any stream capture.  The
 * address is kept per device and context: the first call in a new context of
 * the device (after cudaDeviceReset, for example) looks it up again and must
 * also come before any stream capture.  Keys must lie in [0, grid_num): a key
 * outside it is sorted and written back clamped to 0 or grid_num - 1, without
 * an error (zsph_sort_index reports it through zsph_status).  All calls share
 * the array: calls whose work overlaps on the GPU race.  Errors are reported
 * through zsph_last_error(NULL, ...). */
int zsph_sort_index_noalloc(const zsph_gpu_param_t* gparam, int grid_num, const zsph_tmp_t* tmp, void* stream);
/* cuda_sort_data (single_gpu_sph_src/lib/sort.cu:8-84): grid_start/grid_end
 * from the sorted keys (with the reference's end-of-array rules) and the
 * gather of all eight particle arrays from old_ into new_. */
int zsph_sort_data(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
                   void* stream);
/* hash + sort_index + sort_data in one fused pipeline (bit-identical result). */
int zsph_neighbor_search(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_,
                         const zsph_tmp_t* tmp, void* stream);
/* cuda_boundary_ns (single_gpu_sph_src/equation/delta_ns.cu:5-177): wall
 * pressure, renormalisation matrix, div(v) and renormalised grad(rho) into
 * tmp->dofv_grandrho; new wall (rho, p) into ptc->rhop.  Wall densities are
 * extrapolated before any neighbour reads them (deterministic). */
int zsph_boundary(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream);
/* cuda_govering_ns (delta_ns.cu:179-267): acc and drho/dt into tmp->acc_drhodt. */
int zsph_governing(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream);
/* cuda_prediction / cuda_correction (single_gpu_sph_src/lib/time_int.cu:3-92). */
int zsph_prediction(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream);
int zsph_correction(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream);

/* One full time step (single_gpu_sph_src/deltasph/main.cu:63-88): predictor
 * sub-step and corrector sub-step; the result is in old_ (sorted by the
 * corrector's neighbour search), as in the reference.  new_ is scratch. */
int zsph_step(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
              void* stream);
/* nsteps calls of zsph_step, replayed from one captured CUDA graph. */
int zsph_run(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
             int nsteps, void* stream);

/* List transfer (no reference counterpart; off by default, skin 0.05).  In
 * zsph_step / zsph_run the corrector's neighbour lists are made from the
 * predictor's instead of a second full list build: the predictor also keeps
 * the pairs within 2h + skin*h, the particles that change cell get a full
 * search, and every entry is re-tested against the exact 2h threshold and
 * put back in the reference's visit order.  The lists, and so every result,
 * are those of the full build, bit for bit (particles whose stencil rows
 * can reach stale cell bounds, after a lone last particle, search in full
 * too).  A step whose half-step displacements exceed half the skin, or that
 * kills a particle, builds the corrector's lists in full (the device
 * decides; no host synchronisation).  It applies to single-scene
 * handles with grid factor 1, the delta equations, absolute positions and
 * no rigid body; other steps always build in full.  skin is a multiple of h
 * in [0, 1]; 0 makes every step build in full.  Turning it on allocates
 * about 340 bytes per particle.  On the 4.2 M-particle dam break the
 * transferred lists cost more than the full build (2.5 against 1.6 ms per
 * corrector list), so the plain step keeps the full build. */
int zsph_set_list_transfer(zsph_handle_t* h, int on, float skin);
/* Since the handle was created: steps whose corrector took the transferred
 * lists, steps that built them in full, and particles that got a full search
 * in the transferred steps (synchronises the device; any pointer may be
 * NULL). */
int zsph_list_transfer_info(zsph_handle_t* h, long long* transferred, long long* full_builds,
                            long long* full_searches);

/* Per-particle neighbour counts of a sorted state (after a neighbour
 * search): candidates that pass the reference's distance test
 * (delta_ns.cu:67-68) in the boundary kernel's stencil rows (y < gf,
 * delta_ns.cu:37) and in the governing kernel's rows (y <= gf, :206).
 * Outputs are device int arrays of ptc_num entries (either may be NULL). */
int zsph_neighbor_counts(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int* nb_boundary,
                         int* nb_governing, void* stream);
/* One zsph_step with a CUDA event after every kernel launch: writes each
 * launch's duration in ms into ms[0..cap), their number into *count and the
 * comma-separated kernel names into names (may be NULL). */
int zsph_step_profiled(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
                       void* stream, float* ms, int cap, int* count, char* names, int names_len);
/* As zsph_step_profiled, with events only at the end of each sub-step's
 * neighbour search ("search": hash, scan, scatter, rank + gather) and of its
 * pair kernels ("pair": list build, boundary, governing), so that the
 * durations carry one event's overhead per group instead of one per kernel.
 * No reference counterpart (measurement only). */
int zsph_step_profiled_groups(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_,
                              const zsph_tmp_t* tmp, void* stream, float* ms, int cap, int* count, char* names,
                              int names_len);
/* Number of kernel launches one zsph_step issues. */
int zsph_launches_per_step(zsph_handle_t* h);

/* Synchronises the handle's last stream and returns the accumulated device
 * status bits (ZSPH_FLAG_*), clearing them when clear != 0.  Returns
 * ZSPH_ENAN if the NAN bit is set, ZSPH_ETIMEOUT if the TIMEOUT bit is set,
 * ZSPH_EINVAL if the BAD_KEY bit is set, else ZSPH_OK (or ZSPH_ECUDA). */
int zsph_status(zsph_handle_t* h, int* flags, int clear);
/* Copies the last error message of the handle (or of the library when h is
 * NULL) into buf; returns its length. */
int zsph_last_error(zsph_handle_t* h, char* buf, int len);
/* ---- particle files (legacy VTK, no libVTK) ----------------------------- */

/* Arrays written to a VTK file; the run-time form of the reference's
 * ZSPH_OUTPUT_* compile-time macros (deltasph/CMakeLists.txt:25-31). */
enum {
  ZSPH_OUT_P = 1, ZSPH_OUT_TYPE = 2, ZSPH_OUT_VEL = 4, ZSPH_OUT_ACC = 8,
  ZSPH_OUT_RHO = 16, ZSPH_OUT_HASH = 32, ZSPH_OUT_TABLE = 64,
  ZSPH_OUT_REFERENCE = 1 | 2 | 4 | 8 /* what the deltasph build writes */
};

/* write_vtk (single_gpu_sph_src/io/write_vtk.cu:29-130): legacy VTK, BINARY
 * big-endian, POINTS plus the POINT_DATA arrays selected by flags.  Host
 * arrays in the reference layout; unused ones may be NULL. */
int zsph_write_vtk(const char* path, int ptc_num, const float* pos, const float* vel, const float* rhop,
                   const int* type, const float* acc_drhodt, const int* hash, const int* table, int flags);
/* read_vtk (single_gpu_sph_src/io/read_vkt.cu:3-92): points and the point
 * arrays "p", "rho", "vel", "acc" (double arrays; with accept_float also
 * float arrays, which the reference ignores), "type" (int, required) and
 * "table" (int); missing arrays get the reference's defaults (p 0, rho rho0,
 * vel 0, acc 0, table 0).  ASCII or BINARY; the point count must equal
 * ptc_num. */
int zsph_read_vtk(const char* path, int ptc_num, float rho0, int accept_float, float* pos, float* vel, float* rhop,
                  float* acc_drhodt, int* type, int* table);

/* Output thread pool (io/mul_thread.cu:3-81, deltasph/main.cu:101-142):
 * zsph_writer_submit copies the selected device arrays into one of nthreads
 * pinned host buffers on `stream` (waiting while all buffers are in use) and
 * returns; a worker thread writes output_path/zsph<step>.vtk once the copy has
 * completed.  zsph_writer_destroy finishes pending files and joins. */
typedef struct zsph_writer zsph_writer_t;
int zsph_writer_create(const char* output_path, int ptc_num, int flags, int nthreads, zsph_writer_t** out);
int zsph_writer_submit(zsph_writer_t* w, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int step, void* stream);
int zsph_writer_destroy(zsph_writer_t* w);

/* ---- checkpoint and resume ------------------------------------------------- */

/* No counterpart in the reference, whose only resume state is the case
 * file's start_step/current_step (single_gpu_sph_src/io/read_json.cu:32-35)
 * with an input.vtk that its own output cannot replace (io/write_vtk.cu:56-128
 * writes float arrays and no rho; io/read_vkt.cu:27-39 takes double arrays).
 * A snapshot file holds the non-null arrays of one particle buffer set and of
 * tmp, bit for bit, with the step number and a checksum per array (host byte
 * order).  Saving needs pos, vel, rhop, type, table, grid_start and grid_end
 * (the cell bounds, whose entries from earlier searches can survive a search);
 * null optional arrays are left out.  Loading needs a file of the same
 * ptc_num and grid_num (else ZSPH_EINVAL), checks every array's size and
 * checksum before it writes anything (ZSPH_EIO on a damaged, truncated or
 * foreign file), fills every non-null destination array (ZSPH_EIO if the file
 * lacks one) and returns the saved step in *step.  Buffers loaded from a
 * snapshot of old_ and tmp step on exactly as the saved run does, in the plain
 * and simple equation forms; the precision form's integer cells, a learned
 * corrector's previous values and rigid bodies are held by the handle and are
 * not saved.  zsph_snapshot_save/_load copy device buffers through `stream`
 * and synchronise it; the _host forms take the same structs holding host
 * pointers.  Errors: zsph_last_error(NULL, ...). */
int zsph_snapshot_save(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num, int grid_num,
                       int step, void* stream);
int zsph_snapshot_load(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num, int grid_num,
                       int* step, void* stream);
int zsph_snapshot_save_host(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num,
                            int grid_num, int step);
int zsph_snapshot_load_host(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num,
                            int grid_num, int* step);

/* ---- the reference's driver program ---------------------------------------- */

/* single_gpu_sph_src/deltasph/main.cu:8-147 on this library: reads the case
 * (json_path, then input_path/input.vtk as read_vkt.cu:5 does), selects
 * gpu_id, runs steps start_step .. end_step-1 and writes
 * output_path/zsph<i>.vtk every output_step through the writer pool.
 * ZSPH_COMPAT_SEPARATE issues the reference's twelve launches per step
 * (main.cu:63-88) through the drop-in entry points; ZSPH_COMPAT_FUSED one
 * zsph_step per step.  Or-ing ZSPH_COMPAT_SIMPLE selects the simple-SPH
 * equations (the reference's simplesph program: the same main.cu linked with
 * equation/simple_ns.cu).  *steps_done (may be NULL) receives the number of steps
 * completed.  Nothing is printed; errors are statuses with the message in
 * zsph_last_error(NULL, ...).  When the environment variable ZSPH_METRICS
 * names a file, it receives one JSON line per output step (the reference
 * prints per-step timings to stdout, main.cu:60-95): step, steps and wall
 * seconds since the previous line (the stream synchronised), particle-steps/s,
 * the device status bits and the FP64 conservation sums of the state
 * (zsph_conservation).  The file is rewritten at the start of each run; one
 * that cannot be opened is ZSPH_EIO before any step. */
enum { ZSPH_COMPAT_SEPARATE = 0, ZSPH_COMPAT_FUSED = 1, ZSPH_COMPAT_SIMPLE = 2 };
int zsph_compat_run(const char* json_path, int mode, int* steps_done);

/* ---- Learned-corrector network (no reference counterpart) -----------------
 * A per-particle MLP 32 -> 128 -> 128 -> 4 with SiLU, bf16 weights and fp32
 * accumulation on the fifth-generation tensor cores.  Its fp32 master
 * parameters form one vector of ZSPH_MLP_NPARAM floats:
 *   W1[128][32], b1[128], W2[128][128], b2[128], W3[4][128], b3[4]
 * (weights row-major [out][in]).  Inputs are feature TILES: 128 rows of 32
 * standardized bf16 features, 8 KB per tile, in the tensor-core operand
 * layout (zsph_mlp_pack writes it); rows past the last valid one are zero.
 * Training partials: one row of ZSPH_MLP_NPARTIAL floats per CTA of
 * zsph_mlp_grad, the gradient in parameter order followed by the loss sum. */
enum {
  ZSPH_MLP_IN = 32,
  ZSPH_MLP_HID = 128,
  ZSPH_MLP_OUT = 4,
  ZSPH_MLP_NPARAM = 21252,
  ZSPH_MLP_NPARTIAL = 21256,
  ZSPH_MLP_TILE_ROWS = 128,
  ZSPH_MLP_TILE_BYTES = 8192
};
typedef struct zsph_mlp zsph_mlp_t;
/* Creates the network on the current device with seeded uniform
 * (+-1/sqrt(fan_in)) weights, zero biases and zero Adam moments. */
int zsph_mlp_create(unsigned long long seed, zsph_mlp_t** out);
int zsph_mlp_destroy(zsph_mlp_t* m);
/* Host <-> device copies of the fp32 master parameters (set also refreshes
 * the bf16 weights) and of the Adam moments and step count. */
int zsph_mlp_set_params(zsph_mlp_t* m, const float* params);
int zsph_mlp_get_params(zsph_mlp_t* m, float* params);
int zsph_mlp_set_moments(zsph_mlp_t* m, const float* m1, const float* m2, int step);
int zsph_mlp_get_moments(zsph_mlp_t* m, float* m1, float* m2, int* step);
/* Standardization the learned corrector applies around the network: input
 * feature k enters as (x_k - in_mean[k]) * in_inv_std[k] (32 floats each);
 * output k leaves as y_k * out_std[k] + out_mean[k] (4 floats each). */
int zsph_mlp_set_norm(zsph_mlp_t* m, const float* in_mean, const float* in_inv_std, const float* out_mean,
                      const float* out_std);
int zsph_mlp_get_norm(zsph_mlp_t* m, float* in_mean, float* in_inv_std, float* out_mean, float* out_std);
/* Device rows [n][32] fp32 -> feature tiles: (x - mean) * inv_std rounded to
 * bf16 (mean, inv_std: 32 host floats each); tiles holds ceil(n/128) tiles. */
int zsph_mlp_pack(const float* rows, int n, const float* mean, const float* inv_std, void* tiles, void* stream);
/* out[n][4] (device) = network(tiles), standardized outputs. */
int zsph_mlp_forward(zsph_mlp_t* m, const void* tiles, int n, float* out, void* stream);
/* Gradient of  sum_r w[r] * |net(x_r) - y_r|^2 * inv_wsum  over the tiles
 * tile_ids[0..ntiles) (NULL: tiles 0..ntiles-1); y and w are indexed by
 * tile*128 + row.  Writes *nparts rows of partials (at most the SM count). */
int zsph_mlp_grad(zsph_mlp_t* m, const void* tiles, const float* y, const float* w, const int* tile_ids,
                  int ntiles, float inv_wsum, float* partial, int* nparts, void* stream);
/* One Adam step (fp32, no weight decay) from nparts partial rows, summed in
 * row order; refreshes the bf16 weights. */
int zsph_mlp_adam(zsph_mlp_t* m, const float* partial, int nparts, float lr, float beta1, float beta2, float eps,
                  void* stream);

/* ---- Learned-corrector form of the step (no reference counterpart) --------
 * The predictor sub-step stays the plain one; its governing walk also
 * accumulates 32 non-dimensional neighbour aggregates per fluid particle
 * (lengths in h, speeds in c0, densities in rho0; zeros for walls), among
 * them D = a_n - a_c(prev): the predictor-stage (acc, drho/dt) minus the
 * particle's previous corrector-stage value.  The corrector-stage value is
 * predicted as a_n + D (linear extrapolation over the two half steps) plus
 * the network's residual (accelerations in c0^2/h, density rates in
 * rho0 c0/h), and one tensor-core kernel applies the correction of
 * time_int.cu:50-92 with it in place of the corrector sub-step.  The first
 * step of a run is plain (it has no previous corrector value).  Delta-SPH
 * equations only. */

/* The 32 non-dimensional feature scales of the handle's case. */
int zsph_learn_feature_scales(zsph_handle_t* h, float* scale);
/* The predictor sub-step of zsph_step (search old_ into new_, boundary,
 * governing of new_ with the predicted state written into old_) that also
 * writes the raw features [ptc_num][32] (new_'s sorted order) to the device
 * array `features` (16-byte aligned). */
int zsph_learn_features(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
                        float* features, void* stream);
/* nsteps plain steps (zsph_step); at every `every`-th one the features and
 * the targets (plain corrector minus predictor values) of every particle are
 * kept on the handle as one training snapshot (fluid rows weight 1, others
 * 0), up to `capacity` snapshots (fixed by the first call).  *count: the
 * snapshots held. */
int zsph_learn_collect(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
                       int nsteps, int every, int capacity, int* count, void* stream);
/* Drops the handle's snapshots. */
int zsph_learn_clear(zsph_handle_t* h);

typedef struct {
  int snapshots_train, snapshots_val;
  long long rows_train;        /* fluid rows trained on */
  int epochs, iterations;
  float loss_first, loss_last; /* mean standardized squared error of the first / last epoch */
  /* held-out snapshots, fluid rows: |prediction - corrector| / |corrector|
   * with the network, (_base) with the predictor-stage values alone and
   * (_extrap) with the extrapolation a_n + D alone */
  float val_acc_rel_l2, val_acc_rel_l2_base, val_acc_rel_l2_extrap;
  float val_drho_rel_l2, val_drho_rel_l2_base, val_drho_rel_l2_extrap;
  float seconds;
} zsph_learn_train_stats_t;

/* Trains `net` on the handle's snapshots: sets its standardization from the
 * training snapshots (FP64 moments), then `epochs` passes of Adam over
 * shuffled 128-row tiles (batch_tiles per step, learning rate lr with cosine
 * decay to lr/20, seeded shuffle).  The last val_frac of the snapshots, in
 * collection order, are held out and reported in *stats. */
int zsph_learn_train(zsph_handle_t* h, zsph_mlp_t* net, int epochs, int batch_tiles, float lr,
                     unsigned long long seed, float val_frac, zsph_learn_train_stats_t* stats, void* stream);

typedef struct {
  int steps, learned, plain, judged, fallbacks;
  float err_max, err_mean, err_last; /* judged |a_learned - a_plain| / |a_plain| over fluid particles */
} zsph_learn_run_stats_t;

/* nsteps steps of the learned form.  Every judge_every-th step (0: never)
 * also runs the plain corrector, which judges the network's accelerations
 * (relative L2 over fluid particles) and supplies that step's result; when
 * the error exceeds tol the plain corrector takes over until a judged step
 * passes again.  old_ holds the state afterwards (in the last search's
 * order); the host reads the judge's two sums on judged steps. */
int zsph_run_learned(zsph_handle_t* h, zsph_mlp_t* net, const zsph_ptc_t* old_, const zsph_ptc_t* new_,
                     const zsph_tmp_t* tmp, int nsteps, int judge_every, float tol, zsph_learn_run_stats_t* stats,
                     void* stream);

/* Corrector forms of zsph_run_learned_ex (no reference counterpart).  All
 * run the plain predictor sub-step.
 *   ZSPH_CORR_NETWORK       the network corrector of zsph_run_learned (net required);
 *   ZSPH_CORR_REUSE_LAGGED  no second search and no list build: the corrector's
 *                           governing walk runs on the predictor's neighbour lists
 *                           at the predicted positions (every entry re-tested
 *                           against the exact 2h threshold), with fresh wall
 *                           pressures and the predictor's boundary data
 *                           (renormalised grad rho, div v) (net ignored);
 *   ZSPH_CORR_REUSE_FRESH   the same with a fresh boundary pass on those lists.
 * The list-reuse forms need a single scene, grid factor 1, the delta
 * equations, absolute positions and no rigid body.  Judging and fallback as
 * in zsph_run_learned; err_series (may be null when series_cap is 0)
 * receives the judged relative L2 errors in order, at most series_cap. */
enum { ZSPH_CORR_NETWORK = 0, ZSPH_CORR_REUSE_LAGGED = 1, ZSPH_CORR_REUSE_FRESH = 2 };
int zsph_run_learned_ex(zsph_handle_t* h, zsph_mlp_t* net, const zsph_ptc_t* old_, const zsph_ptc_t* new_,
                        const zsph_tmp_t* tmp, int nsteps, int judge_every, float tol, int corrector,
                        float* err_series, int series_cap, zsph_learn_run_stats_t* stats, void* stream);

/* ---- Batched form (no reference counterpart) ------------------------------
 * One handle over nscenes independent cases (grid_size_factor 1, delta-SPH
 * equations).  Scene s owns the particles [P_s, P_s + ptc_num_s) of the
 * handle's buffers, P_s = the sum of the earlier scenes' ptc_num (scenes
 * stored one after another, each in its own particle order), and its own
 * cells; every kernel launch of zsph_step / zsph_run covers all scenes, so
 * a step is one graph whatever the number of scenes.  A particle that
 * leaves its scene's grid is parked in that scene's first cell.  Per scene
 * the results are those of a handle created for that scene alone. */
int zsph_create_batch(const zsph_gpu_param_t* scenes, const int* grid_num, int nscenes, zsph_handle_t** out);
/* Batched handle in persistent mode (no reference counterpart): zsph_step
 * and zsph_run advance every scene with one cooperative launch per step whose
 * CTAs stay resident and pass each stage (search, list build, boundary,
 * governing with the integration) through a grid barrier instead of a kernel
 * boundary.  The stages run the same device code as the step's separate
 * launches, so the results are bit-identical with them.  zsph_run captures
 * the launch in its CUDA graph when the driver accepts a cooperative launch
 * in a capture, and otherwise issues one launch for all its steps.  Every
 * barrier wait is bounded (about a second); a wait that runs out sets
 * ZSPH_FLAG_TIMEOUT, every CTA leaves the kernel, and zsph_status returns
 * ZSPH_ETIMEOUT.  on = 0 returns to the separate launches. */
int zsph_set_batch_persistent(zsph_handle_t* h, int on);
/* CTAs of the persistent launch, and whether zsph_run replays it from a
 * graph (1), issues it directly (-1) or has not run yet (0). */
int zsph_persistent_info(zsph_handle_t* h, int* ctas, int* graph);
/* Self-test of the bounded barrier: one persistent launch whose barrier
 * waits for an arrival that never comes, each wait limited to spin_limit
 * polls; returns ZSPH_ETIMEOUT (and clears the flag) when the bound works. */
int zsph_persistent_barrier_test(zsph_handle_t* h, int spin_limit, void* stream);

/* ---- Autotuner (no reference counterpart) ----------------------------------
 * Times every candidate launch shape of the grid-factor-1 step -- cells
 * (warps) per CTA of the neighbour-list build {2, 4}, cells (segments) a
 * list-build warp handles together per round {2, 3, 4}, minimum resident
 * CTAs per SM of the governing kernel {1, 6, 8} (its register budget), steps
 * per graph replay of zsph_run {1, 4} (36 candidates) -- for trial_steps steps each on the
 * handle's buffers, restores old_ and the carried tmp arrays after every
 * trial, and keeps the fastest for the handle's later zsph_run calls. */
typedef struct {
  int list_cells_per_cta, governing_min_ctas, steps_per_graph;
  float ms_per_step;  /* of the chosen shapes */
  float ms_default;   /* of the untuned shapes */
  int candidates;
  int list_segments;  /* list build: cells handled together per round {2, 3, 4} (0: the default, 4) */
} zsph_tune_t;
int zsph_autotune(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_ptc_t* new_, const zsph_tmp_t* tmp,
                  int trial_steps, zsph_tune_t* out, void* stream);
/* Applies launch shapes chosen earlier (a zsph_autotune result kept by the
 * caller, e.g. across restarts of the same case) without timing anything:
 * list_cells_per_cta, list_segments, governing_min_ctas and steps_per_graph
 * from the candidate sets above, 0 for each one's default (2 warps, 4
 * segments, 1 CTA, 1 step); the time fields are ignored.  ZSPH_EINVAL for any
 * other value. */
int zsph_set_launch_shapes(zsph_handle_t* h, const zsph_tune_t* shapes);

/* ---- Precision form (no reference counterpart) ----------------------------
 * zsph_set_precision(h, 1): a particle's position is held as its integer grid
 * cell (one int per particle, kept on the handle for old_ and new_ and moved
 * by the search) plus the FP32 offset from the cell's corner, which the pos
 * arrays then hold instead of absolute coordinates.  Pair distances are
 * formed as cell difference * grid_size + offset difference, and zsph_step /
 * zsph_run integrate offsets and move cells.  Needs grid_size_factor 1, the
 * delta-SPH equations and grid dimensions up to 1023; the fused step entry
 * points only (zsph_step, zsph_run). */
int zsph_set_precision(zsph_handle_t* h, int on);
/* Loads absolute FP64 positions (host, [ptc_num][3]) into old_ as cell +
 * offset (the precision form must be on). */
int zsph_precise_load(zsph_handle_t* h, const zsph_ptc_t* old_, const double* pos, void* stream);
/* Absolute FP64 positions of old_ (host, [ptc_num][3]); also valid with the
 * precision form off (then the FP32 positions widened). */
int zsph_precise_positions(zsph_handle_t* h, const zsph_ptc_t* old_, double* pos, void* stream);

/* FP64 global sums over the fluid particles of old_ (and the attached body):
 * mass, volume sum(m/rho), momentum, kinetic energy, potential energy
 * -m g z, internal energy of the linear equation of state
 * m c0^2 (ln(rho/rho0) + rho0/rho - 1). */
typedef struct {
  double mass, volume, momentum[3], kinetic, potential, internal;
  double body_kinetic, body_potential;
} zsph_conservation_t;
int zsph_conservation(zsph_handle_t* h, const zsph_ptc_t* old_, zsph_conservation_t* out, void* stream);

/* ---- 6DOF rigid body coupled to the fluid (no reference counterpart) -------
 * The particles of type 2 whose original index (table[i] + i) lies in
 * [first, first + count) form one rigid body of the given mass.  They act
 * as dummy walls (density and pressure extrapolated from the fluid,
 * delta_ns.cu:61-131) that move with the body.  After every fused
 * sub-step's governing kernel the fluid's pressure force on each body
 * particle is summed in FP64 into the body's force and torque about its
 * centre of mass, the body is advanced in FP64 by the same predictor-
 * corrector as the fluid (angular acceleration as
 * Test_6DOF/equation/acc_alpha.cpp:20-33, quaternion rate as
 * Test_6DOF/equation/time_int.cpp:14-15), and its particles are placed from
 * its pose.  Inertia: Test_6DOF/equation/rigid_info.cpp:18-39 (about the
 * particles' centroid, mass shared equally).  Works with and without the
 * precision form. */
typedef struct {
  int first, count;         /* original particle indices of the body */
  double mass;              /* kg */
  double pos[3];            /* centre of mass (output: the particles' centroid) */
  double vel[3], omega[3];  /* linear and angular (world frame) velocity */
  double q[4];              /* orientation (w, x, y, z) */
  double force[3], torque[3]; /* output: the last fluid force and torque */
  double inertia[9];        /* output: body-frame inertia about the centre of mass */
} zsph_rigid_t;
/* Attaches a body to the handle using the particles' current positions in
 * old_ (the body frame is the given orientation); sets the body particles'
 * velocities from vel and omega.  Up to 16 bodies with disjoint particle
 * ranges: a body whose first index equals an attached body's replaces it,
 * any other is added (ZSPH_EINVAL on an overlapping range or a 17th body). */
int zsph_rigid_attach(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_rigid_t* body, void* stream);
/* Current state of the first attached body. */
int zsph_rigid_get(zsph_handle_t* h, zsph_rigid_t* body);
/* Number of attached bodies, and the current state of body `index` (in
 * attach order). */
int zsph_rigid_count(zsph_handle_t* h, int* count);
int zsph_rigid_get_body(zsph_handle_t* h, int index, zsph_rigid_t* body);
/* Contact of the bodies with the walls and with each other (no counterpart
 * in the reference, whose Test_6DOF bodies never touch anything): a body
 * particle and a non-fluid particle of the walls or of another body closer
 * than `distance` (m, at most the 2h support; dx makes bodies touch at their
 * surfaces) push apart along the pair's normal with
 * max(0, stiffness (distance - r) - damping v_n) newtons, v_n the normal
 * relative velocity; the force enters the body's FP64 force and torque sums
 * beside the fluid's.  stiffness 0 (the default) turns contact off.
 * Grid factor 1 only. */
int zsph_rigid_contact(zsph_handle_t* h, double stiffness, double damping, double distance);

/* Plain device-memory helpers for callers without their own CUDA runtime
 * binding (the reference driver calls cudaMalloc/cudaMemcpy directly,
 * deltasph/main.cu:41-45).  kind: 1 host->device, 2 device->host,
 * 3 device->device; the copy is complete on return. */
int zsph_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream);
int zsph_device_malloc(void** p, size_t bytes);
int zsph_device_free(void* p);
int zsph_device_synchronize(void);

/* Library version string. */
const char* zsph_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ZSPH_H */
