// Internal declarations shared by the sm_100a kernels and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/zsph.h"

namespace zsph {

constexpr int kSearchBlock = 256;  // threads per CTA for the streaming (HBM-bound) kernels
constexpr int kScanItems = 8;      // cells per thread in the cell-offset scan
constexpr int kScanTile = kSearchBlock * kScanItems;
constexpr int kBigSegment = 256;   // cells holding more particles than this are pre-sorted by a CTA
constexpr int kBigListCap = 4096;  // at most this many such cells are pre-sorted per sub-step
constexpr int kPairBlock = 128;    // threads per CTA for the neighbour-list and pair kernels
constexpr int kMaxNb = 128;        // neighbour-list capacity per particle (overflow -> direct path)

// Constants of one case, passed by value to every kernel.  Mirrors
// gpu_param_t plus the values the kernels derive from it once on the host.
struct KParams {
  zsph_gpu_param_t p;
  int n;                 // particles
  int G;                 // cells
  int XY;                // grid_xdim * grid_ydim
  float r2lo, r2hi;      // rr2 < r2lo => q <= 2 for sure; rr2 > r2hi => q > 2 for sure
  float r2max;           // q = sqrtf(rr2)/h <= 2 exactly when rr2 <= r2max (IEEE, monotone)
  float inv_h;
  float inv_gs;          // 1 / grid_size
  float c_fr;            // -5 * adh / h2, the factor of grad W / r
  int stage_windows;     // 1: pair kernels stage neighbour windows in shared memory (TMA bulk copies)
  int equations;         // ZSPH_EQ_DELTA or ZSPH_EQ_SIMPLE
  // Precision form (null otherwise): a particle's position is its grid cell
  // (hx | hy << 10 | hz << 20) plus the FP32 offset from that cell's corner
  // held in pos.  c3o belongs to the buffer searched from (old_), c3n to the
  // buffer searched into (new_).
  int* c3o;
  int* c3n;
  // Rigid body attached (null otherwise): the governing kernel writes, for
  // each type-2 particle, the pressure acceleration from its fluid
  // neighbours alone (the fluid's force on the body per unit particle mass).
  float4* rigid_f;
  // Batched form (null otherwise): independent scenes, scene s owning the
  // particles [pbase[s], pbase[s+1]) and the cells [cbase[s], cbase[s+1]);
  // kernels resolve their scene and use its parameters (scene_kp).
  const struct SceneDev* scenes;
  const int* scene_pbase;
  const int* scene_cbase;
  int nscenes;
  // Launch shapes chosen by zsph_autotune (0 = the default): cells (warps)
  // per CTA of the list build (2, 4) and the governing kernel's minimum
  // resident CTAs per SM (1, 6, 8), i.e. its register budget.
  int tune_cw;
  int tune_minb;
  int tune_segs;         // list build: cells (segments) per round, 2, 3 or 4 (0 = 4)
  // Learned form's list-reuse correctors (null otherwise): each particle's
  // grid row (y cell index) at the current positions, which decides the
  // boundary stencil's asymmetric rows y in [-GF, GF) (delta_ns.cu:37).
  const int* cur_cy;
  // List transfer (plain step, set for the predictor's governing launch
  // only; null otherwise): the fused prediction also writes each particle's
  // predicted position to xfer_pos4 and sets *xfer_flag when the corrector
  // must build its lists in full (a displacement above sqrt(disp2max), a
  // non-finite position, or a position the corrector's hash will kill).
  float4* xfer_pos4;
  int* xfer_flag;
  float disp2max;  // largest squared half-step displacement the transfer allows
  float r2skin;    // predictor list build: squared outer radius of the skin lists
};

// Original-index range [first, first + count) of one rigid body.
struct BodyRange {
  int first, count;
};

// One scene of the batched form: its case constants as KParams holds them.
struct SceneDev {
  zsph_gpu_param_t p;  // grid_hash_min/max: the scene's cells in batch coordinates
  int XY;
  float r2lo, r2hi, r2max, inv_h, inv_gs, c_fr;
};

// scene owning index v: the last s with base[s] <= v (base ascending, nscenes + 1 entries)
__device__ __forceinline__ int scene_of(const int* base, int nscenes, int v) {
  int lo = 0, hi = nscenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(base + mid) <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// the kernel parameters of scene s (batch-wide particle and cell counts)
__device__ __forceinline__ KParams scene_kp(const KParams& kp, int s) {
  KParams r = kp;
  const SceneDev& d = kp.scenes[s];
  r.p = d.p;
  r.XY = d.XY;
  r.r2lo = d.r2lo;
  r.r2hi = d.r2hi;
  r.r2max = d.r2max;
  r.inv_h = d.inv_h;
  r.inv_gs = d.inv_gs;
  r.c_fr = d.c_fr;
  return r;
}
__device__ __forceinline__ KParams kp_of_particle(const KParams& kp, int i) {
  return (kp.scenes && i < kp.n) ? scene_kp(kp, scene_of(kp.scene_pbase, kp.nscenes, i)) : kp;
}
__device__ __forceinline__ KParams kp_of_cell(const KParams& kp, int c) {
  return (kp.scenes && c < kp.G) ? scene_kp(kp, scene_of(kp.scene_cbase, kp.nscenes, c)) : kp;
}

// packed integer cell coordinates of the precision form
constexpr int kCellBits = 10;
constexpr int kCellMask = (1 << kCellBits) - 1;
__host__ __device__ __forceinline__ int pack_cell(int hx, int hy, int hz) {
  return hx | (hy << kCellBits) | (hz << (2 * kCellBits));
}
__host__ __device__ __forceinline__ int3 unpack_cell(int c) {
  return make_int3(c & kCellMask, (c >> kCellBits) & kCellMask, (c >> (2 * kCellBits)) & kCellMask);
}

// 256-bit global load / store of one 32-byte record (sm_100 v8 vector
// access; the address must be 32-byte aligned).
__device__ __forceinline__ void ld_rec(const float4* p, float4& a, float4& b) {
  asm("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}
__device__ __forceinline__ void st_rec(float4* p, float4 a, float4 b) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x), "f"(a.y), "f"(a.z),
               "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

struct ShadowRec {
  float4 pr, vp;
};

// Packed per-particle shadows of the sorted state, written by the list build
// (each particle's own record, with a wall's new density and pressure), or by
// k_pack where no list build runs:
// one 32-byte record per particle, rec[2i] = pr = {x, y, z, +-rho} with the
// sign bit set for non-fluid particles (type != 1) and rec[2i+1] = vp =
// {vx, vy, vz, p}, so that a pair kernel fetches a neighbour's record with
// one 256-bit load instead of two 16-byte loads.  rec comes from cudaMalloc
// (256-byte aligned), so every record is 32-byte aligned.
struct Shadow {
  float4* rec;  // [2n]
  __device__ __forceinline__ float4& pr(int i) const { return rec[2 * i]; }
  __device__ __forceinline__ float4& vp(int i) const { return rec[2 * i + 1]; }
  __device__ __forceinline__ ShadowRec load(int i) const {
    ShadowRec r;
    ld_rec(rec + 2 * i, r.pr, r.vp);
    return r;
  }
};

// List transfer: the corrector's neighbour lists made from the predictor's
// (transfer.cu).  Device scratch, allocated when a handle enables it.
constexpr int kSkinCap = 16;  // predictor skin entries per particle (2h < r <= 2h + skin)
constexpr int kXtra = 8;      // corrector candidates handed to a particle by the full-search set
struct Xfer {
  uint16_t* nb2;     // corrector lists, blocked like Scratch::nb
  uint8_t* nb_cnt2;  // [n]
  uint16_t* sk;      // [ceil(n/32)*32 * kSkinCap] predictor skin lists, blocked by 32-particle groups
  uint8_t* sk_cnt;   // [n] (255 = overflow)
  float4* pos4;      // [n] predicted positions in predictor order; .w = the particle's corrector slot
  int* xl;           // [n * kXtra] predictor indices handed to a particle by the full-search set
  int* xcnt;         // [n] entries in xl (zeroed before the corrector's search)
  int* hashP;        // [n] predictor search's hash and cell bounds, copied before the corrector's search
  int* gsP;          // [G]
  int* geP;          // [G]
  int* flag;         // [1] nonzero: the corrector builds its lists in full this step
  uint8_t* fullb;    // [n] 1: the corrector slot gets a full search
  int* alist;        // [n] the corrector slots with a full search (unordered)
  int* acount;       // [1] entries in alist (zeroed before the corrector's search)
  unsigned long long* stats;  // [3] steps transferred, steps that built in full, full searches
};

// The kernels move the float2 particle arrays (rhop, tmp_rhop) with 8-byte
// accesses: every float array of a particle buffer must start on an 8-byte
// boundary (cudaMalloc gives 256).  Checked on the host before any launch.
inline bool ptc_aligned8(const zsph_ptc_t& p) {
  const void* a[] = {p.pos, p.vel, p.rhop, p.tmp_pos, p.tmp_vel, p.tmp_rhop};
  for (const void* q : a)
    if (reinterpret_cast<uintptr_t>(q) & 7u) return false;
  return true;
}

constexpr int kMiscWords = 16;  // Scratch::misc
constexpr int kMiscWalls = 8;   // misc word holding the wall list's length
constexpr int kMiscFluidEpoch = 9;  // misc word: the search epoch whose cfe stamps are valid (0: none)

// Programmatic dependent launch: the kernel's grid may start while the
// previous kernel in the stream drains (a CUDA graph keeps the relation as
// a programmatic edge).  Such a kernel calls pdl_wait() before anything
// else: it returns once the previous grid has completed and its writes are
// visible (and at once when there is no such grid).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Device scratch owned by a handle; allocated once in zsph_create.
struct Scratch {
  int* cnt;          // [G]   per-cell counts (kept zero between uses)
  int* cell_lb;      // [G+1] exclusive prefix of counts: first sorted slot of each cell
  int* key;          // [n]   unsorted cell keys
  int* ticket;       // [n]   arrival rank inside the key's cell
  int* perm;         // [n]   scattered original positions (stable after ranking)
  int* val;          // [n]   carried values for zsph_sort_index
  int* tile_sum;     // [tiles]
  int* tile_off;     // [tiles]
  int* tile_last;    // [tiles] last occupied cell of each tile (-1 if none)
  int* misc;         // [kMiscWords] 0: tiles done, 1: last key, 2: count of last key, 3: big-cell list length,
                     //       4: largest key (one-pass scan), 5: one-pass scan tile counter, 6: one-pass scan epoch,
                     //       7: the fused scatter's finished-CTA counter (crowded cells),
                     //       kMiscWalls: entries in wl (zeroed before each list build),
                     //       kMiscFluidEpoch: the epoch of the cfe stamps (0 after the drop-in gather)
  unsigned long long* tile_state;  // [tiles] one-pass scan: (tag << 32) | prefix value, tag from the epoch
  int* big_list;     // [kBigListCap]
  uint16_t* nb;      // [ceil(n/32)*32 * kMaxNb] neighbour lists, blocked by 32-particle groups (equations.cu)
  uint8_t* nb_cnt;   // [n] neighbour count (255 = overflow)
  int* wl;           // [n] sorted slots of the non-fluid particles, appended by the list build (unordered)
  int* cfe;          // [G] per cell: the search epoch (misc[6]) in which the fused gather put a fluid particle there
  int* flags;        // [1]   ZSPH_FLAG_* bits
  Shadow sh;
  Xfer xf;           // list transfer scratch (null pointers when the handle has none)
};


// Learned-corrector inputs written by the predictor-stage governing walk
// (k_governing<GF, 1, true>): kFeat non-dimensional neighbour aggregates per
// fluid particle (zeros for walls).  Feature k of particle i is
// raw = sum_k * scale[k]; the network reads (raw - mean) * inv_std as bf16
// in the tensor-core tile layout.
constexpr int kFeat = 32;
struct FeatOut {
  float* raw;              // [n][kFeat] raw features, or null
  unsigned char* tiles;    // ceil(n/128) tiles of standardized bf16 features, or null
  float4* acc_copy;        // copy of the predictor-stage (acc, drho/dt), or null
  const float4* acc_prev;  // previous corrector-stage (acc, drho/dt) in the search's source order
  float4* d_out;           // [n] D = predictor-stage value - previous corrector value (sorted order)
  float scale[kFeat];
  float mean[kFeat];
  float inv_std[kFeat];
};

// Optional per-launch event markers (profiling): after each kernel launch the
// launcher records the next event, so event k-1 -> k brackets launch k.  With
// `external` set the launches are being captured into a graph and the marks
// become event-record nodes of that graph.  With `groups` set only the ends of
// the launch groups are marked: the neighbour search (after rank_gather,
// labelled "search") and the pair kernels (after governing, labelled "pair").
struct Prof {
  cudaEvent_t* ev = nullptr;
  int cap = 0;
  int n = 0;
  const char** names = nullptr;
  bool external = false;
  bool groups = false;
};

inline void mark(Prof* pf, const char* name, cudaStream_t st) {
  if (!pf || pf->n >= pf->cap) return;
  if (pf->groups) {
    const std::string k(name);
    if (k == "rank_gather") name = "search";
    else if (k == "governing" || k == "governing_feat") name = "pair";
    else return;
  }
  pf->names[pf->n] = name;
  if (pf->external) cudaEventRecordWithFlags(pf->ev[pf->n++], st, cudaEventRecordExternal);
  else cudaEventRecord(pf->ev[pf->n++], st);
}

struct Handle {
  KParams kp;
  Scratch s;
  int device = 0;
  int tiles = 0;
  cudaStream_t last_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  zsph_ptc_t graph_old{}, graph_new{};
  zsph_tmp_t graph_tmp{};
  cudaStream_t graph_stream = nullptr;
  std::string err;
  struct LearnState* learn = nullptr;  // learned-corrector data and scratch (learn.cu)
  int* c3buf[2] = {nullptr, nullptr};  // precision form: cells of old_ / new_ (precise.cu)
  struct RigidState* rigid = nullptr;  // attached rigid body (precise.cu)
  SceneDev* scene_tab = nullptr;       // batched form: scene table and bases (device)
  int* scene_base = nullptr;           // [2][nscenes + 1]: particle bases, then cell bases
  int graph_steps = 1;                 // steps per replay of zsph_run's graph (zsph_autotune)
  // batched form in one persistent launch per step (zsph_set_batch_persistent)
  int persistent = 0;
  unsigned* pbar = nullptr;            // the persistent kernel's grid-barrier words [2]
  unsigned spin_limit = 1u << 22;      // polls per barrier wait (about a second)
  int persist_graph = 0;               // 1: zsph_run replays a captured persistent launch; -1: capture refused
  // list transfer (zsph_set_list_transfer): on/off and the skin as a multiple of h
  int xfer_on = 0;
  float xfer_skin = 0.05f;
};

// learn.cu: frees the handle's learned-corrector state
void learn_destroy(Handle* h);
// precise.cu: frees the precision-form and rigid-body state
void precise_destroy(Handle* h);
// precise.cu: FP64 force/torque sum, body update and placement after a
// fused sub-step's governing kernel (mode 1 predictor, 2 corrector)
cudaError_t rigid_substep(Handle* h, const zsph_ptc_t& from, const zsph_ptc_t& to, const zsph_tmp_t& t, int mode,
                          cudaStream_t st);

// api.cu: one sub-step of the fused path (search `from` into `to`, boundary
// on `to`, governing of `to` with the integration written into `from`)
cudaError_t run_substep(Handle* h, const zsph_ptc_t& from, const zsph_ptc_t& to, const zsph_tmp_t& t, int mode,
                        cudaStream_t st, Prof* pf, const FeatOut* feat);

// mlp.cu
struct Mlp {
  float* w = nullptr;   // fp32 master parameters (ZSPH_MLP_NPARAM)
  float* m1 = nullptr;  // Adam moments
  float* m2 = nullptr;
  void* w1 = nullptr;   // bf16 weights [128][32], [128][128], [16][128]
  void* w2 = nullptr;
  void* w3p = nullptr;
  int step = 0;
  // input / output standardization of the learned corrector
  float in_mean[kFeat], in_inv_std[kFeat];
  float out_mean[4], out_std[4];
};
cudaError_t launch_mlp_correct(const Mlp& m, const KParams& kp, const void* tiles, const zsph_ptc_t& ptc,
                               float4* acc, const float4* dprev, float4 oa, float4 ob, int* flags, cudaStream_t st);
cudaError_t launch_mlp_forward(const Mlp& m, const void* tiles, int n, float* out, int* flags, cudaStream_t st);
cudaError_t launch_mlp_grad(const Mlp& m, const void* tiles, const float* y, const float* w, const int* ids,
                            int ntiles, float inv_wsum, float* partial, int* nparts, int* flags, cudaStream_t st);
cudaError_t launch_mlp_adam(Mlp& m, const float* partial, int nparts, float lr, float b1, float b2, float eps,
                            cudaStream_t st);
cudaError_t launch_mlp_pack(const float* rows, int n, const float* mean, const float* inv_std, void* tiles,
                            cudaStream_t st);
int mlp_sm_count();

// api.cu: message returned by zsph_last_error(NULL, ...)
void record_library_error(const std::string& msg);
// Unique id of the calling thread's current CUDA context (never reused within
// a process), or 0 when there is none yet or the driver does not offer it
// (device_context.cu).  Host state that belongs to one context is kept per
// device with this id and set up again when it differs; with 0 it is set up
// again on every call.
unsigned long long current_context_id();

// search.cu
cudaError_t launch_hash(const KParams& kp, int* flags, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp, cudaStream_t st);
cudaError_t launch_sort_index(const KParams& kp, const Scratch& s, int tiles, const zsph_tmp_t& tmp, cudaStream_t st);
cudaError_t launch_sort_data(const KParams& kp, const Scratch& s, int tiles, const zsph_ptc_t& o, const zsph_ptc_t& w,
                             const zsph_tmp_t& tmp, cudaStream_t st);
cudaError_t launch_search(const KParams& kp, const Scratch& s, int tiles, const zsph_ptc_t& o, const zsph_ptc_t& w,
                          const zsph_tmp_t& tmp, cudaStream_t st, Prof* pf = nullptr);
// packed shadows + exact cell ranges of a caller-sorted state (drop-in pair entry points)
cudaError_t launch_pack(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                        cudaStream_t st);

// packed shadows of a state in its current order (no cell ranges)
cudaError_t launch_pack_shadows(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, cudaStream_t st);

// equations.cu
// Learned form's corrector variants on the lists of the predictor's search
// (ptc: the predicted state in that sorted order): shadows repacked, wall
// (rho, p) at the predicted positions, optionally a fresh boundary pass
// (else tmp.dofv_grandrho keeps the predictor's values), then governing with
// mode 0 (acc_drhodt only) or 2 (correction written in place into ptc).
// cy: n ints of scratch for the particles' current y cell indices.
cudaError_t launch_corrector_reuse(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                                  bool fresh_boundary, int mode, int* cy, cudaStream_t st);
cudaError_t launch_boundary(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                            cudaStream_t st, Prof* pf = nullptr);
// one-time kernel attributes (shared-memory windows above 48 KB); call before launches
cudaError_t init_pair_kernels();
// mode 0: acc_drhodt only; 1: + prediction into out; 2: + correction into out
// feat (mode 1, delta equations only): also write the learned-corrector inputs
cudaError_t launch_governing(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                             int mode, const zsph_ptc_t& out, cudaStream_t st, Prof* pf = nullptr,
                             const FeatOut* feat = nullptr);
cudaError_t launch_nblist(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                          cudaStream_t st);
// List transfer (equations.cu): the predictor's list build with skin lists
// plus its boundary pass; the corrector's transferred lists (full build when
// the transfer's conditions failed) plus its boundary pass on s.xf's lists.
cudaError_t launch_xfer_pred_lists(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                                   cudaStream_t st, Prof* pf);
cudaError_t launch_xfer_corr_lists(const KParams& kp, const Scratch& s, const zsph_ptc_t& cur, const zsph_tmp_t& tmp,
                                   cudaStream_t st, Prof* pf);
// Batched form: nsteps full steps of every scene in one cooperative launch
// (equations.cu, k_batch_persistent); bar: two zeroed device words of the
// grid barrier, kept between launches.  spin_limit bounds each barrier wait;
// extra > 0 (self-test) adds arrivals that never come.
cudaError_t launch_batch_persistent(const KParams& kp, const Scratch& s, const zsph_ptc_t& o, const zsph_ptc_t& w,
                                    const zsph_tmp_t& t, unsigned* bar, int nsteps, unsigned spin_limit, int extra,
                                    cudaStream_t st);
// CTAs of that launch (all resident at once)
cudaError_t persistent_grid(int* grid);
// Rigid bodies: adds to kp.rigid_f of every body particle of ptc (the state
// the lists were built for) the contact force per unit particle mass of its
// non-fluid neighbours that are not of its own body, within `dist` (<= 2h):
// max(0, kn (dist - r) - cn v_n) along the pair's normal.
cudaError_t launch_rigid_contact(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                                 const BodyRange* ranges, int nb, float kn, float cn, float dist, cudaStream_t st);
cudaError_t launch_nb_counts(const KParams& kp, const Scratch& s, int* nb_boundary, int* nb_governing,
                             cudaStream_t st);
cudaError_t launch_integrate(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                             int correction, cudaStream_t st);

}  // namespace zsph

// the opaque C types of include/zsph.h
struct zsph_handle : public zsph::Handle {};
struct zsph_mlp : public zsph::Mlp {};
