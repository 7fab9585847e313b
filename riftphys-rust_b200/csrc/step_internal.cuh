// step_internal.cuh -- per-tick scratch buffers, the tick context, and the small set of
// device-wide primitives (radix sort, scan, select) the pipeline uses.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "world_gpu.h"

namespace rp {

#define RP_CUDA(x)                                                                      \
  do {                                                                                  \
    cudaError_t e__ = (x);                                                              \
    if (e__ != cudaSuccess)                                                             \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e__) + \
                               " at " __FILE__ ":" + std::to_string(__LINE__));         \
  } while (0)

// Kernel launches issued by this library (exact: every launch site adds its count; each
// device-wide sort / scan / select adds the kernels it runs).
// Counting also checks the launch: a bad configuration is reported at its own line instead of
// surfacing later as the "last error" of an unrelated call.
extern unsigned long long g_launches;
inline void count_launch(unsigned n, const char* file, int line) {
  g_launches += n;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " at " + file + ":" + std::to_string(line));
}
#define RP_COUNT_LAUNCH(n) ::rp::count_launch((n), __FILE__, __LINE__)

// d_stats slots
enum : int {
  STAT_ERR = 0,          // RPHYS_STATERR_* bits
  STAT_WARM_MATCHED = 1,
  STAT_BOUNCE = 2,
  STAT_SWEEPS = 3,       // max sweeps over islands
  STAT_RESID = 4,        // f32 bits of the max residual (non-negative: integer max is order-free)
  STAT_SLEEPING = 5,
  STAT_LEVELS = 6,
  STAT_MAXBATCH = 7,
  STAT_NISL = 8,
  STAT_ROWSWEEPS = 9,    // velocity row updates this tick (rows x sweeps, summed over islands)
  STAT_GROUPS_SHARED = 10,
  STAT_GROUPS_GLOBAL = 11,
  STAT_MAX_GROUP_ROWS = 12,
  STAT_MAX_GROUP_BODIES = 13,
  STAT_ISLANDS_CAPPED = 14,
  STAT_PRED_USED = 15,   // rows that started from the learned prediction
  STAT_ROWS_CAPPED = 16, // residual mode: rows of the islands still above the tolerance at the cap
  STAT_RES_HIST = 17,    // 6 slots: solve islands by their last sweep's residual (res_bin)
  STAT_COUNT = 23
};
// The residual histogram's bin of an island's last-sweep residual r (m/s): <= 1e-4, 1e-3, 1e-2,
// 1e-1, 1, and above 1 (or NaN). The CPU restatement bins with the same f32 comparisons.
__host__ __device__ inline uint32_t res_bin(float r) {
  if (r <= 1.0e-4f) return 0u;
  if (r <= 1.0e-3f) return 1u;
  if (r <= 1.0e-2f) return 2u;
  if (r <= 1.0e-1f) return 3u;
  if (r <= 1.0f) return 4u;
  return 5u;
}



// Stages timed with CUDA events on the world's stream when profiling is on.
enum Phase : int {
  PH_FORCES = 0, PH_AABB, PH_BROAD, PH_NARROW, PH_TERRAIN, PH_CONTACTS, PH_ISLANDS, PH_ROWS, PH_SCHED,
  PH_WARM_MATCH, PH_VEL_SOLVE, PH_WARM_CACHE, PH_VEL_SHOCK, PH_BALLISTIC, PH_INTEGRATE, PH_POS_ITER,
  PH_POS_SHOCK, PH_STAGE6,
  // parts of vel_solve (nested inside it; named "vel_solve.*"): the rows' staging before the
  // classes fork, the packed groups, the big islands, and each single-island bucket on its stream
  PH_VEL_PREP, PH_VEL_PACKED, PH_VEL_BIG, PH_VEL_ISL0, PH_VEL_ISL1, PH_VEL_ISL2, PH_VEL_ISL3, PH_VEL_ISL4,
  PH_VEL_ISL5, PH_COUNT
};
static const char* const kPhaseNames[PH_COUNT] = {
    "forces", "aabb_sweep", "broadphase", "narrow_pairs", "terrain", "contacts", "islands", "rows", "schedule",
    "warm_match", "vel_solve", "warm_cache", "vel_shock", "ballistic", "integrate", "pos_iter", "pos_shock", "stage6",
    "vel_solve.prep", "vel_solve.packed", "vel_solve.big", "vel_solve.island128", "vel_solve.island256",
    "vel_solve.island384", "vel_solve.island512", "vel_solve.island768", "vel_solve.island1152"};

struct Profiler {
  bool on = false;
  cudaEvent_t ev[PH_COUNT][2] = {};
  bool used[PH_COUNT] = {};
  double ms[PH_COUNT] = {};
  uint64_t calls[PH_COUNT] = {};
  void begin(int p, cudaStream_t st) {
    if (!on) return;
    if (!ev[p][0]) { cudaEventCreate(&ev[p][0]); cudaEventCreate(&ev[p][1]); }
    cudaEventRecord(ev[p][0], st);
  }
  void end(int p, cudaStream_t st) {
    if (!on) return;
    cudaEventRecord(ev[p][1], st);
    used[p] = true;
  }
  // after the stream is idle: fold this tick's events into the totals
  void collect() {
    if (!on) return;
    for (int p = 0; p < PH_COUNT; ++p) {
      if (!used[p]) continue;
      float t = 0.0f;
      if (cudaEventElapsedTime(&t, ev[p][0], ev[p][1]) == cudaSuccess) { ms[p] += t; calls[p] += 1; }
      used[p] = false;
    }
  }
  void reset() { for (int p = 0; p < PH_COUNT; ++p) { ms[p] = 0; calls[p] = 0; used[p] = false; } }
};

// Growth doubles (a buffer that tracks a rising contact count regrows rarely). Inside a tick the
// world's stream is set in g_alloc_stream and growth goes through the stream-ordered allocator,
// whose pool keeps freed memory (release threshold set at world creation): no device-wide
// synchronisation in the middle of a tick. Contents are not kept across growth.
extern thread_local cudaStream_t g_alloc_stream;
template <class T>
void DBuf<T>::ensure(size_t n) {
  if (n <= cap) return;
  size_t c = n < 16 ? 16 : 2 * n;
  if (g_alloc_stream) {
    if (p) RP_CUDA(cudaFreeAsync(p, g_alloc_stream));
    p = nullptr;
    RP_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), c * sizeof(T), g_alloc_stream));
  } else {
    if (p) cudaFree(p);
    p = nullptr;
    RP_CUDA(cudaMalloc(&p, c * sizeof(T)));
  }
  cap = c;
}
// Sets g_alloc_stream for the scope of one tick.
struct AllocStreamScope {
  cudaStream_t prev;
  explicit AllocStreamScope(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
  ~AllocStreamScope() { g_alloc_stream = prev; }
};
template <class T>
void DBuf<T>::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

struct WorldGpu::Scratch {
  // per body
  DBuf<float4> pre_lin, pre_ang, orig_pos, orig_rot, pred_pos, pred_rot, split_l, split_a;
  DBuf<float> Iw;
  DBuf<uint8_t> constrained, loaded, ballistic, touching;
  DBuf<uint32_t> uf, uf2, body_level, isl_of_root, root_mark;
  // per collider
  DBuf<float4> amin, amax, smin, smax;
  DBuf<float> sweep;
  DBuf<uint32_t> u32a, u32b, sap_ids, over_ids, sap_key, sap_key2, sap_ord, sap_cnt, sap_off, ov_cnt, ov_off, counts;
  DBuf<float> minx;
  // pairs and narrowphase
  DBuf<unsigned long long> pairs, pairs2;
  DBuf<uint8_t> flag8;
  DBuf<float4> p_pt, p_n, t_pt, t_n;
  DBuf<uint32_t> p_cnt, t_cnt, pstart, bcnt, boff;
  DBuf<int4> t_win;
  DBuf<uint32_t> t_ncell, t_celloff, t_icnt, t_ioff;
  DBuf<float4> t_cp, t_cn, t_sp, t_sn;  // terrain points: packed, and 8 slots per (collider, cell) item
  // contacts
  DBuf<uint32_t> c_a, c_b;
  DBuf<float4> c_pt, c_n;  // c_pt.w = depth, c_n.w = impulse
  // rows (solver.rs:47-87 ContactConstraint, the fields the configured path reads)
  DBuf<uint2> r_ab;
  DBuf<uint32_t> r_flags;
  DBuf<float2> r_inv;
  DBuf<float4> r_ra, r_rb, r_n, r_t1, r_t2, r_mu, r_la;
  DBuf<float> acc_jn;
  DBuf<float2> acc_jt;
  DBuf<int> wm_idx;
  // schedules
  DBuf<uint32_t> row_isl, row_isl2, rows_sched, rows_sched2, isl_start, isl_cnt, level, lvl_cnt, lvl_off,
      lvl_start, ord_main, ord_vs, ord_ps, lvl_off_vs, lvl_start_vs, lvl_off_ps, lvl_start_ps, nlev, nlev_vs, nlev_ps,
      tmp32, tmp32b;
  DBuf<unsigned long long> key64, key64b;
  DBuf<uint32_t> lvl_hist, row_level;
  DBuf<uint32_t> lv_key, lv_key2, lv_val, lv_val2, lv_pred, lv_level, lv_np1, lv_lead;  // parallel level schedule
  DBuf<uint4> col_mask;                                                        // coloured order: colours per body
  DBuf<uint32_t> col_nlev, col_ord;
  DBuf<uint32_t> isl_final;
  DBuf<unsigned long long> wh_meta, wh_ch0;                                    // per-world hashes of a batch
  DBuf<uint32_t> wh_wbs, wh_jr, wh_roots;                                                    // per solve island: last residual (bits)
  DBuf<uint32_t> row_islid, row_lisl, li_flag, li_pre, g_nisl;                 // islands inside solve groups
  DBuf<uint32_t> pp_rows, pp_key, pp_gs, pp_gc, ord_pp, lvl_off_pp, lvl_start_pp, nlev_pp;  // position pass (joints)
  DBuf<uint32_t> cls_cnt, cls_list;                                            // solve groups by class
  DBuf<unsigned long long> sap_key64, sap_key64b;                              // batched worlds: (world, min x)
  DBuf<uint32_t> sap_w, gp_cnt, gp_off;
  DBuf<float4> big_x, big_j;                                                   // big-island row stream
  DBuf<float> feat, pred3, targets;                                            // learned warm start
  // W6 bounce passes: per contact the time-of-impact data, then the passes' scratch
  DBuf<float4> toi_a;
  DBuf<float2> toi_b;
  DBuf<uint32_t> w6_rest_cnt, w6_rest_min, w6_rest_max, w6_parent, w6_slot, w6_rows, w6_comp_rows, w6_comp_start,
      w6_row_comp, w6_cur, w6_ctr;
  DBuf<uint8_t> w6_involved, w6_direct, w6_in_set, w6_has_pseudo, w6_pool;
  DBuf<double> w6_acc;
  DBuf<float4> w6_pl, w6_pa;
  DBuf<float> w6_target, w6_sup_acc, w6_pseudo_u;
  // the wire snapshot
  DBuf<uint32_t> wire_flag, wire_off;
  DBuf<uint8_t> wire_buf;
  // ray casts
  DBuf<float4> ray_in, ray_pt, ray_n;
  DBuf<uint8_t> feat_valid;
  DBuf<float4> pred_used, s_pred;
  // solve groups (islands packed for one CTA each) and their shared-memory residents
  DBuf<uint32_t> g_small_rows, g_small_pre, g_big, g_big_pre, g_of_isl, g_key, g_key2, g_start, g_cnt, g_class,
      g_iota, g_perm, g_sz_sorted, g_pre_sorted, body_grp, gb_key, gb_key2, gb_list, gb_tmp, gb_start, gb_cnt, body_local;
  // rows in schedule order (coalesced per level) for the shared-memory solve
  DBuf<uint2> s_loc;                      // local body index of A / B (0xFFFFFFFF: cannot move)
  DBuf<uint32_t> s_flags;
  DBuf<float2> s_inv;
  DBuf<float4> s_ra, s_rb, s_n, s_t1, s_t2, s_mu, s_va, s_vb, s_wa, s_wb;
  DBuf<float> s_jn;
  DBuf<float2> s_jt;
  DBuf<int> s_wm;
  // position pass
  DBuf<float4> pc_la, pc_lb;
  // warm cache build
  DBuf<uint8_t> wflag;
  DBuf<uint32_t> woff, wpos;
  // hash
  DBuf<uint8_t> hbuf;
  DBuf<uint32_t> hcv, jh_sz, jh_off, jh_has, jh_pos;
  // primitives' temporary storage
  DBuf<uint8_t> cub_tmp;
  DBuf<uint4> kept_k;
  DBuf<float4> kept_a, kept_b;
  Profiler prof;
};

// The heightfield as the terrain kernel reads it (HeightField, terrain.rs:13-21); h == nullptr: none.
struct HFView { const float* h; uint32_t nx, nz; float sx, sz, ox, oz, min_y, max_y; };

struct StepCtx {
  float dt;
  f3 g, up;
  uint32_t np = 0, nc = 0, nisl = 0, nref_isl = 0, nsched = 0;
  uint32_t g_small = 0;  // solve groups [0, g_small) are packed groups of small islands
  HFView hf{nullptr, 0, 0, 1, 1, 0, 0, 0, 0};
  uint32_t hf_mat = 4;
};

// ---- primitives (step_prims.cu)
void select_flagged_iota(WorldGpu::Scratch& S, int n, const uint32_t* flags, uint32_t* out, uint32_t* d_count,
                         cudaStream_t st);
uint32_t select_flagged_u64(WorldGpu::Scratch& S, const unsigned long long* in, const uint8_t* flags,
                            unsigned long long* out, uint32_t n, cudaStream_t st);
uint32_t select_flagged_u32(WorldGpu::Scratch& S, const uint32_t* in, const uint8_t* flags, uint32_t* out,
                            uint32_t n, cudaStream_t st);
void sort_pairs_u32(WorldGpu::Scratch& S, const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout,
                    uint32_t n, int bit0, int bit1, cudaStream_t st);
void sort_pairs_u64(WorldGpu::Scratch& S, const unsigned long long* kin, unsigned long long* kout, const uint32_t* vin,
                    uint32_t* vout, uint32_t n, int bit0, int bit1, cudaStream_t st);
void sort_keys_u64(WorldGpu::Scratch& S, const unsigned long long* kin, unsigned long long* kout, uint32_t n,
                   cudaStream_t st);
uint32_t exclusive_scan_total(WorldGpu::Scratch& S, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t st);
void exclusive_scan(WorldGpu::Scratch& S, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t st);

void run_front(WorldGpu& W, StepCtx& ctx);
void run_solve(WorldGpu& W, StepCtx& ctx);

}  // namespace rp
