// Shared device/host definitions for the B200 mill sub-step: the per-mill descriptor, the
// per-sub-step uniform block, the output record, and the scalar arithmetic of the reference
// (glam 0.29 Vec2 semantics, pbf.rs kernels) in f32 without fused multiply-add (the library is
// built with -fmad=false; division and square root are IEEE).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/millgpu.h"

#define MG_HD __host__ __device__ __forceinline__

namespace mg {

constexpr float PI_F = 3.14159265358979323846f;
constexpr float TAU_F = 6.28318530717958647692f;
constexpr float GRAVITY = -9.81f;
constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr int MAX_LIFTERS = 64;
// Per-ball sweeps (drag, buoyancy): warps taking balls and the poll interval of a waiting ball.
constexpr uint32_t DEFAULT_SWEEP_WARPS = 32;
// ... for single-mill handles, whose helper blocks take the sweeps' other work meanwhile (fewer
// waiting warps keep more issue slots for the ball on the dependency chain; measured fastest)
constexpr uint32_t DEFAULT_SWEEP_WARPS_SINGLE = 20;
// Largest block of the frame kernel (32 warps); per-warp scratch (the merge slot maps) is sized for it.
constexpr uint32_t MAX_BLOCK_THREADS = 1024;
constexpr uint32_t MAX_BLOCK_WARPS = MAX_BLOCK_THREADS / 32;
// Threads per mill block when the options leave it open (measured fastest on B200, single mill
// and batches alike).
constexpr uint32_t DEFAULT_BLOCK_THREADS = 1024;
// Thread blocks that run one mill's per-ball stages in a single-mill launch: the mill's own block
// plus helper blocks (at most MAX_MILL_BLOCKS; DEFAULT_MILL_BLOCKS unless the caller sets it).
constexpr uint32_t MAX_MILL_BLOCKS = 16;
constexpr uint32_t DEFAULT_MILL_BLOCKS = 16;
constexpr uint32_t DEFAULT_SPIN_NS = 64;
// Bounds of the device's waits: polls of a ball waiting for an earlier ball in a per-ball sweep
// (about a second at the default poll interval), and clock cycles of a wait between a mill's
// block and its helper blocks (about 10 s at 2 GHz).
constexpr uint32_t SPIN_LIMIT = 1u << 24;
constexpr long long WIDE_TIMEOUT_CYCLES = 20000000000LL;
constexpr int MAX_BOUNDARY_POINTS = 1024;

// ---------------------------------------------------------------- scalar helpers (f32::max etc.)
MG_HD float fmax_r(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  return a > b ? a : b;
}
MG_HD float fmin_r(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  return a < b ? a : b;
}
MG_HD float clamp_r(float x, float lo, float hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
MG_HD bool finite_f(float x) { return x - x == 0.0f; }
MG_HD bool isnan_f(float x) { return x != x; }
MG_HD int32_t f2i_sat(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}
MG_HD uint32_t f2u_sat(float f) {
  if (f != f || f <= 0.0f) return 0;
  if (f >= 4294967296.0f) return UINT32_MAX;
  return (uint32_t)f;
}
MG_HD int32_t sat_add(int32_t a, int32_t b) {
  int64_t s = (int64_t)a + (int64_t)b;
  if (s > INT32_MAX) return INT32_MAX;
  if (s < INT32_MIN) return INT32_MIN;
  return (int32_t)s;
}
MG_HD float powi3(float x) { return x * (x * x); }
MG_HD float powi5(float x) { float x2 = x * x; float x4 = x2 * x2; return x * x4; }
MG_HD float powi6(float x) { float x2 = x * x; float x4 = x2 * x2; return x2 * x4; }
MG_HD float powi8(float x) { float x2 = x * x; float x4 = x2 * x2; return x4 * x4; }

// Transcendentals as the f32 rounding of the f64 function (the oracle does the same on the host).
MG_HD float expf_r(float x) { return (float)exp((double)x); }
MG_HD float sinf_r(float x) { return (float)sin((double)x); }
MG_HD float cosf_r(float x) { return (float)cos((double)x); }
MG_HD float atan2f_r(float y, float x) { return (float)atan2((double)y, (double)x); }
MG_HD float log10f_r(float x) { return (float)log10((double)x); }

// ---------------------------------------------------------------- glam::Vec2 semantics
struct V2 {
  float x, y;
  MG_HD V2() : x(0.0f), y(0.0f) {}
  MG_HD V2(float a, float b) : x(a), y(b) {}
  MG_HD V2(float2 f) : x(f.x), y(f.y) {}
  MG_HD float2 f2() const { return make_float2(x, y); }
  MG_HD V2 operator+(V2 o) const { return V2(x + o.x, y + o.y); }
  MG_HD V2 operator-(V2 o) const { return V2(x - o.x, y - o.y); }
  MG_HD V2 operator-() const { return V2(-x, -y); }
  MG_HD V2 operator*(float s) const { return V2(x * s, y * s); }
  MG_HD V2 operator/(float s) const { return V2(x / s, y / s); }
  MG_HD V2& operator+=(V2 o) { x += o.x; y += o.y; return *this; }
  MG_HD V2& operator-=(V2 o) { x -= o.x; y -= o.y; return *this; }
  MG_HD V2& operator*=(float s) { x *= s; y *= s; return *this; }
  MG_HD float dot(V2 o) const { return (x * o.x) + (y * o.y); }
  MG_HD float len2() const { return dot(*this); }
  MG_HD float len() const { return sqrtf(dot(*this)); }
  MG_HD bool finite() const { return finite_f(x) && finite_f(y); }
  MG_HD V2 normalize() const { float rcp = 1.0f / len(); return *this * rcp; }
  MG_HD V2 normalize_or_zero() const {
    float rcp = 1.0f / len();
    if (finite_f(rcp) && rcp > 0.0f) return *this * rcp;
    return V2();
  }
};
MG_HD V2 operator*(float s, V2 v) { return V2(s * v.x, s * v.y); }
MG_HD float cross2(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }
MG_HD V2 rotate(V2 v, V2 u) { return V2(v.x * u.x - v.y * u.y, v.x * u.y + v.y * u.x); }

// ---------------------------------------------------------------- pbf.rs:119-181 kernels
MG_HD float poly6(float r2, float h) {
  if (r2 >= h * h || r2 < 0.0f) return 0.0f;
  float h2 = h * h;
  float term = h2 - r2;
  return 4.0f / (PI_F * powi8(h)) * term * term * term;
}
MG_HD V2 spiky_grad(V2 delta, float r, float h) {
  if (r <= 1e-9f || r >= h) return V2();
  float coeff = -30.0f / (PI_F * powi5(h)) * (h - r) * (h - r);
  return (delta / r) * coeff;
}
MG_HD float cohesion_kernel(float r, float h) {
  if (r <= 0.0f || r >= h) return 0.0f;
  float coeff = 35840.0f / (209.0f * PI_F * powi8(h));
  float term = powi3(h - r) * powi3(r);
  if (r <= 0.5f * h) return coeff * (2.0f * term - powi6(h) / 64.0f);
  return coeff * term;
}
MG_HD float adhesion_kernel(float r, float h) {
  if (r <= 0.5f * h || r >= h) return 0.0f;
  float coeff = 35840.0f / (163.0f * PI_F * powi8(h));
  return coeff * powi3(h - r) * powi3(r);
}

// ---------------------------------------------------------------- uniform inputs of one sub-step
// Everything here is mill-uniform and computed on the host in the reference's arithmetic
// (drum-angle trig, lifter frames, boundary-point offsets, squeeze-film prefactors).
struct FilmConsts { double r, c1, c2, prefactor; };

struct StepUniform {
  // drum (geometry.rs)
  float drum_radius, drum_omega;
  uint32_t lifter_count;
  float lifter_height, lifter_base_half, lifter_top_half;
  float lifter_cos[MAX_LIFTERS], lifter_sin[MAX_LIFTERS];
  float drum_angle, drum_angle_next;
  V2 to_local_next, to_world_next;  // from_angle(-angle_next), from_angle(angle_next)
  V2 to_local0;                     // from_angle(-angle)
  float dt;
  uint32_t pbf_iterations, dem_iterations;
  uint32_t run_fluid, run_dem, dem_external;
  MgMediaParams media;
  MgSlurryParams slurry;
  // ball boundary points for adhesion and viscosity groups (pbf.rs:190-219)
  uint32_t boundary_count;
  V2 boundary_offset[MAX_BOUNDARY_POINTS];
  // squeeze films (mac/lubrication.rs; pbf.rs:544-625)
  FilmConsts pair_film, wall_film;
  uint32_t cg_fp64;
  uint32_t want_momentum;  // accumulate CouplingImpulses::fluid_momentum_change (coupling.rs:49-51)
  uint32_t sweep_warps;    // warps taking balls in the per-ball sweeps
  uint32_t spin_ns;        // poll interval of a waiting ball
  double now_s;            // the sub-step's SubAngles::now_s and alpha (the stress fold)
  float alpha;
  uint32_t fold_stress;    // 1: fold each sub-step's impacts into the stress accumulator (Simulation::step)
  uint32_t spin_limit;     // polls after which a waiting ball gives up (ERR_BUDGET)
  uint32_t skip_done_ball; // tests only: the drag sweep never flags this ball done (NONE: none)
  uint32_t sweep_order;    // per-ball sweeps: 0 claim balls by dependency level, 1 by index
};

// The per-sub-step part of the uniform block (drum angle and its rotations, dt), one per sub-step
// of a launch; the kernel copies it into the mill's StepUniform before each sub-step.
struct SubAngles {
  float drum_angle, drum_angle_next, dt, pad;
  V2 to_local_next, to_world_next, to_local0;
  double now_s;  // Simulation::sim_time when the sub-step's impacts are folded (stress.rs now_s)
  float alpha;   // its EMA weight, 1 - exp(-dt / 1 s) in f32 (lib.rs:516-537)
  float pad2;
};

// stress.rs:80-99 StressAccum without its debounce map (which is the hash table below): the EMA
// rates, the cumulative sums and the update count, in f64 as the reference keeps them.
struct StressState {
  double count_rate[4], se_hat_rate[4], hist_rate[MG_SE_BINS], above_rate_j[6];
  double cum_wall_j, cum_above_j[6];
  unsigned long long updates;
};

// ---------------------------------------------------------------- per-sub-step outputs
struct StepOut {
  MgFluidStepStats fs;
  MgDemStepStats ds;
  MgStepCounters ctr;
  float fluid_momentum[2];
  uint32_t clamp_hits;
  uint32_t n_impacts;
  uint32_t err;
  uint32_t pad;
  // per-stage device cycles (clock64 deltas at the stage barriers); slots 0-14 follow the
  // reference's stage_timing.rs STAGE_NAMES, 15-18 split the DEM step, 19 is drag alone, 20-31
  // split the sweeps further (see capi.STAGE_NAMES)
  unsigned long long stage[40];
};

enum : uint32_t {
  ERR_EDGES = 1u << 0,
  ERR_PAIRS = 1u << 1,
  ERR_CELLS = 1u << 2,
  ERR_RECORDS = 1u << 3,
  ERR_ITEMS = 1u << 4,
  ERR_GROUPS = 1u << 5,
  ERR_LINKS = 1u << 6,
  ERR_IMPACTS = 1u << 7,
  ERR_BUDGET = 1u << 8,
  ERR_WIDE = 1u << 9,  // a mill's helper blocks and its own block stopped waiting for each other
  ERR_STRESS = 1u << 10,  // the impact debounce table had no free slot
};

// ---------------------------------------------------------------- a spatial grid's buffers
struct GridBuf {
  int2* pkey;           // per point cell key (cap_points)
  uint32_t* cell_start; // cap_cells + 1
  uint32_t* cursor;     // cap_cells + 1 (scratch)
  uint32_t* indices;    // cap_points
  int2* keys;           // sparse: unique sorted keys (cap_points)
  uint32_t cap_points, cap_cells;
};

// The grid header a build produces (lives in shared memory).
struct GridHdr {
  float cell;
  int32_t dense;
  int32_t min_cx, min_cy;
  int32_t width, height;
  uint32_t ncells;   // dense: width*height; sparse: unique keys
  uint32_t npoints;  // valid (finite) points
};

// Control block of a single-mill launch with helper blocks (mill_wide.cuh): the mill's block
// publishes phases, the helper blocks count the phases they finished. Zeroed before each launch.
struct WideCtl {
  uint32_t seq;      // phases published so far
  uint32_t phase;    // the last published phase
  uint32_t done;     // helper-block phases finished, over the launch
  uint32_t counter;  // a phase's count summed over the helper blocks
  GridHdr hdr;       // the grid the phase searches
  const float2* vin; // the vectors a phase reads and writes (joint operator)
  float2* vout;
  // the next sub-step's fluid steps 0-3 on helper block 1 (WIDE_FLUID_PREP): its dt, and what the
  // mill's block takes over from them (their error bits, kept apart from the mill's error word
  // while the mill's block runs the DEM step; the fluid grid's header, edge count, density
  // iterations, the helper's cycles of steps 0-2 and of step 3)
  float prep_dt;
  uint32_t prep_err;
  GridHdr prep_hdr;
  uint32_t prep_edges, prep_iters;
  unsigned long long prep_cycles[2];
  // the finished sub-step's fluid tail (mean shear rate, speed clamp and their kinetic-energy
  // terms), run by helper block 1 before the steps 0-3 above when tail_out is set: that sub-step's
  // output record, its speed cap and the fluid kinetic energy before the viscosity solve
  StepOut* tail_out;
  float tail_vmax;
  double tail_ke;
  // the work the helper blocks do beside the drag sweep (WIDE_BESIDE_DRAG): which parts run
  // (BESIDE_*), the viscosity the Morris weights use; helper block 1 publishes the group grid's
  // header (beside_grid_seq = the phase's sequence number once it is built); the other helpers
  // count their finished buoyancy item shares (beside_buoy_blocks); helper block 1 leaves the
  // buoyancy records' count and whether it found a claim order
  uint32_t beside_tasks;
  float beside_mu;
  uint32_t beside_grid_seq;
  uint32_t beside_buoy_blocks;
  GridHdr beside_hdr;
  uint32_t beside_nrec, beside_order_ok;
  GridHdr beside_link_hdr;      // the squeeze links' ball grid (cell 2 r + reach)
  uint32_t beside_link_over;    // balls whose squeeze-link candidates did not fit their slots
  // helpers done with their boundary-group shares (beside_group_blocks); helper block 1 then
  // compacts the groups and sorts them by fluid particle, leaving the count (beside_ngroups) and
  // whether it did (beside_groups_ok)
  uint32_t beside_group_blocks, beside_ngroups, beside_groups_ok;
  // the drag sweep's item lists, records and claim order, listed by the helper blocks while the
  // mill's block runs steps 5-6 (WIDE_DRAG_LISTS): helper block 1 publishes the drag grid's header
  // (drag_grid_seq = 1 once built), the other helpers count their finished shares of the item
  // lists and the per-ball pre-sums (drag_blocks), helper block 1 then leaves whether it found a
  // claim order
  uint32_t drag_grid_seq, drag_blocks, drag_order_ok;
  GridHdr drag_hdr;
};
enum : uint32_t { BESIDE_VISC = 1u, BESIDE_BUOY = 2u };

// ---------------------------------------------------------------- per-mill descriptor
struct MillDev {
  uint32_t nf, nb;
  uint32_t cap_nf, cap_nb;
  uint32_t cap_edges, cap_pairs, cap_groups, cap_links, cap_recs, cap_items, cap_impacts;
  uint32_t* guess_valid_dev;  // 1 once a viscous warm start of length nf is stored in fguess
  uint32_t* err;              // sticky error bits (ERR_*) of this mill
  // materials
  float f_mass, f_h, f_rho0;
  float b_r, b_m, b_I, b_rtrue;
  // state
  float2 *fx, *fv, *fguess;
  float* fdye;
  float2 *bx, *bv;
  float *bth, *bom;
  // coupling impulses (coupling.rs:37-63)
  float2* imp;
  float* ang;
  // fluid workspace
  float2 *x0, *dp, *push_ex, *coh_dv, *adh_dv, *dv_tmp;
  float *density, *lambda, *wall_val, *f_tmp, *mu_eff;
  int32_t* wall_bin;
  uint32_t* nbr_off;  // cap_nf + 1
  uint32_t* nbrs;     // cap_edges
  float* visc_w;      // cap_edges
  float2* visc_dir;   // cap_edges
  GridBuf gA, gB, gBall;
  // records: overlap push (i, b, J, L, M) and adhesion (fluid, dv)
  uint32_t *rec_i, *rec_b;
  float2 *rec_J, *rec_M;
  float* rec_L;
  uint32_t* rec_cnt;  // cap_nf + 1 (per fluid particle counts / offsets)
  // per-ball item lists (adhesion / drag / buoyancy / groups), cap_items per ball
  uint32_t* item_j;
  float2* item_v;
  float *item_w, *item_w2;
  uint32_t* item_n;  // cap_nb + 1
  uint32_t *bk_start, *bk_cur, *bk_order;  // bucket-sort scratch
  // viscosity: groups, links, CG vectors
  uint32_t *g_fluid, *g_ball;
  float *g_c, *g_l2;
  float2* g_lc;
  uint32_t* g_off;  // per ball group offsets (cap_nb + 1)
  uint32_t *fg_start, *fg_list;  // per fluid group lists
  uint32_t *l_ball, *l_other;
  float2* l_n;
  float* l_c;
  uint32_t* l_off;  // per ball own-link offsets (cap_nb + 1)
  uint32_t *lo_start, *lo_list;  // per ball "other" link lists
  float2 *cg_x, *cg_b, *cg_r, *cg_z, *cg_p, *cg_ap, *cg_lv;
  float *cg_diag, *cg_inv;
  float2* ball_v0;
  float* drag_pre;  // per ball: the drag sweep's geometry-only quantities (8 floats)
  float* ball_w0;
  // dem workspace
  float2 *bx0, *bvpre;
  float *bth0, *bompre, *lam_bw;
  float2* bxs;    // ball positions at the start of the projection sweep
  float* bmove;   // per ball largest squared distance from bxs during the projection sweep
  double* f_cw;  // per-ball coupling work of the predict step
  uint32_t *rec_off, *rec_pred, *ball_done;  // per-ball sweep records (cap_nb + 1, cap_recs, cap_nb)
  uint32_t* slot;  // per-warp fluid -> item maps of the in-order merges (warps of all the mill's blocks x cap_nf, all NONE at rest)
  // single-mill handles with helper blocks: the item lists the helpers fill beside the drag sweep
  // (boundary groups in gi_*, buoyancy items in bi_*, cap_items per ball like item_*), the
  // buoyancy records (b_rec_*: offsets, fluid index, ball, predecessor ball), the helpers'
  // bucket-sort scratch and the buoyancy sweep's claim order; null otherwise
  uint32_t* gi_j;
  float2* gi_v;
  float *gi_w, *gi_w2;
  uint32_t *bi_j, *bi_n;
  float2* bi_v;
  float* bi_w;
  uint32_t *b_rec_off, *b_rec_i, *b_rec_b, *b_rec_pred;
  uint32_t *hb_start, *hb_cur, *hb_order;
  uint32_t* b_order;
  uint32_t* d_order;  // the drag sweep's claim order when the helper blocks listed its items
  // squeeze-link candidates the helpers list beside the drag sweep (geometry only; which of them
  // are links depends on the balls' velocities after the sweeps): per ball i, its partners j > i
  // within reach in slots [i K, i K + K) (K = min(nb + 1, 512)) with their normals and film
  // coefficients, their count, and the wall candidate (in range, normal, coefficient)
  uint32_t* lk_j;
  float2* lk_n;
  float* lk_c;
  uint32_t *lk_cnt, *lk_winr;
  float2* lk_wn;
  float* lk_wc;
  uint32_t *pair_i, *pair_j;
  float* lam_bb;
  uint32_t* pr_list;  // pairs within reach of touching at the start of the projection
  uint32_t* pair_cnt;  // per cell pair counts (cap cells + 1)
  // sweep replay (mill_replay.cuh): predecessors, levels, active contacts of the contact sweeps
  uint32_t *dm_pa, *dm_pb, *dm_lvl, *lev_start, *lev_cur, *lev_items;
  uint32_t *act_i, *act_j, *act_flag;
  float *act_l, *act_w1, *act_w2, *act_t;
  int32_t* act_bin;
  MgImpactRecord* act_rec;
  uint32_t smem_balls;  // balls whose state fits the launch's dynamic shared memory (0: global)
  uint32_t smem_bytes;  // the launch's dynamic shared memory (staged ball state, then sweep scratch)
  // the impact-energy accumulator (stress.rs:110-171) on the device: its state, the debounce
  // table (keys (ball, partner) with (0, 0) free, the time each was last counted; st_cap a power
  // of two) and, when set, where the launch leaves a copy of the state for the host
  StressState* stress;
  uint2* st_key;
  double* st_time;
  uint32_t st_cap;
  StressState* stress_copy;
  uint32_t helpers;     // helper blocks of this launch (set by the kernel; 0 in batches)
  uint32_t test_extra_helpers;  // tests only: helper blocks the mill's block waits for but were not launched
  long long wide_wait_cycles;   // the mill block's bound on a wait for its helper blocks (clock cycles)
  WideCtl* wide;        // their control block
  // outputs
  StepOut* out;             // one per sub-step of the launch
  MgImpactRecord* impacts;  // cap_impacts per sub-step of the launch
};

}  // namespace mg
