// C ABI of the library (include/millgpu.h): simulation handles over device-resident mill state.
// The host prepares the mill-uniform inputs (drum rotations, lifter frames, boundary offsets,
// squeeze-film constants) and folds the per-sub-step outputs the device writes into the
// Simulation bookkeeping of lib.rs:470-565 (EMA power and torque, f64 energy budget, the stress
// accumulator of stress.rs with its debounce table), exactly in sub-step order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <deque>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "mill_kernels.h"
#include "mill_params.h"
#include "mill_stress.cuh"

using namespace mg;

namespace {

thread_local std::string g_err;

int fail_global(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// ------------------------------------------------------------------ stress.rs:28-171
// The accumulator itself runs on the device (mill_stress.cuh, folded after every sub-step of
// Simulation::step); the handle keeps a copy of its state, refreshed after every launch.
double stress_total_rate(const StressState& st) {
  return st.count_rate[0] + st.count_rate[1] + st.count_rate[2] + st.count_rate[3];
}

// ------------------------------------------------------------------ device arena
struct Arena {
  size_t off = 0;
  char* base = nullptr;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += std::max<size_t>(n, 1) * sizeof(T);
    return p;
  }
};

constexpr uint32_t MAX_SUB = 64;

}  // namespace

struct MgSim {
  MgParams params;
  MgOptions opt{};
  std::string err;
  // Simulation scalars (lib.rs:82-119)
  float drum_angle = 0.0f;
  double sim_time = 0.0;
  float power = 0.0f, torque = 0.0f, collision_rate = 0.0f, dissipated_power = 0.0f, max_disp = 0.0f;
  uint32_t clamp_hits_frame = 0;
  MgFluidStepStats last_fluid{};
  MgDemStepStats last_dem{};
  MgStepCounters last_ctr{};
  MgEnergyBudget budget{};
  double e0 = 0.0;
  StressState stress{};  // the device accumulator's state after the last launch
  // device state
  cudaStream_t stream = nullptr;
  // a light handle (a request-server job): it borrows the server's stream, takes its arena from
  // the device's stream-ordered memory pool and keeps its host blocks in pageable memory; it is
  // only ever advanced by the server's batched launches
  bool light = false;
  // thread blocks the arena's merge slot maps are sized for: a plain handle's single-mill launches
  // may spread its per-ball stages over this many blocks (batch and server mills use one)
  uint32_t mill_blocks_cap = 1;
  uint32_t nf = 0, nb = 0, cap_nf = 0, cap_nb = 0;
  MgBallMaterial bmat{};
  MgFluidMaterial fmat{};
  void* dmem = nullptr;
  size_t dbytes = 0;
  MillDev md{};
  MillDev* d_md = nullptr;
  StepUniform* h_uni = nullptr;
  StepUniform* d_uni = nullptr;
  SubAngles* h_ang = nullptr;
  SubAngles* d_ang = nullptr;
  StepOut* h_out = nullptr;
  MgImpactRecord* h_imp = nullptr;
  MgMetrics* d_metrics = nullptr;  // mg_metrics output (in the arena)
  void* surf_mem = nullptr;        // mg_fluid_surface scratch (allocated on first use)
  uint32_t* h_surf = nullptr;      // pinned staging of the surface header and output head
  SurfDev surf{};
  uint32_t guess_valid_host = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_kernel_ms = 0.0f;
  uint64_t launches = 0;
  uint64_t ctr_tot[10] = {};
  uint64_t ctr_n = 0;
  uint64_t stage_tot[40] = {};
};

namespace {

int fail(MgSim* s, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (s) s->err = buf;
  g_err = buf;
  return code;
}

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return fail(s, MG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

uint32_t cap_items_for() { return 256; }

// Sizes the device arena for nf fluid particles and nb balls. Capacities: fluid edges 64 nf + 1024,
// ball pairs 64 nb + 1024, boundary groups 256 nb, squeeze links nb min(nb + 1, 512) + 1024,
// 256 coupling items per ball, 4 nb + 256 impact records per sub-step, up to MAX_SUB sub-steps per
// launch; a bound that is exceeded sets its ERR_* bit and the call returns MG_ERR_CAPACITY.
int alloc_state(MgSim* s, uint32_t nf, uint32_t nb) {
  if (s->dmem && nf <= s->cap_nf && nb <= s->cap_nb) {
    s->nf = nf;
    s->nb = nb;
    s->md.nf = nf;
    s->md.nb = nb;
    return MG_OK;
  }
  // the stress accumulator's debounce table survives a new arena: its live keys are carried over
  std::vector<uint2> old_keys;
  std::vector<double> old_times;
  if (s->dmem) {
    old_keys.resize(s->md.st_cap);
    old_times.resize(s->md.st_cap);
    CK(cudaMemcpyAsync(old_keys.data(), s->md.st_key, sizeof(uint2) * s->md.st_cap, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(old_times.data(), s->md.st_time, sizeof(double) * s->md.st_cap, cudaMemcpyDeviceToHost,
                       s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (s->light) cudaFreeAsync(s->dmem, s->stream);
    else cudaFree(s->dmem);
    s->dmem = nullptr;
  }
  uint32_t cf = std::max(nf, 1u), cb = std::max(nb, 1u);
  MillDev m{};
  m.cap_nf = cf;
  m.cap_nb = cb;
  m.cap_edges = 64u * cf + 1024u;
  m.cap_pairs = 64u * cb + 1024u;
  m.cap_items = cap_items_for();
  m.cap_groups = cb * m.cap_items;
  // squeeze links: every pair of balls within 2r + 8 dx plus the wall, bounded by nb per ball
  m.cap_links = cb * std::min<uint32_t>(cb + 1u, 512u) + 1024u;
  m.cap_recs = std::max({8u * cf + 1024u, m.cap_groups, m.cap_links, 2u * m.cap_pairs + cb + 64u});
  m.cap_impacts = 4u * cb + 256u;
  // debounce table: eight slots per impact record a sub-step can hold, a power of two
  m.st_cap = 1u;
  while (m.st_cap < 8u * m.cap_impacts) m.st_cap <<= 1;
  const uint32_t fcells = 2u * cf + 513u, bcells = 2u * cb + 513u;
  const uint32_t nbig = std::max(cf, cb) + 2u;
  // pass 1: measure, pass 2: carve
  for (int pass = 0; pass < 2; ++pass) {
    Arena a;
    a.base = pass ? (char*)s->dmem : nullptr;
    m.guess_valid_dev = a.take<uint32_t>(1);
    m.err = a.take<uint32_t>(1);
    m.stress = a.take<StressState>(1);
    m.st_key = a.take<uint2>(m.st_cap);
    m.st_time = a.take<double>(m.st_cap);
    m.fx = a.take<float2>(cf); m.fv = a.take<float2>(cf); m.fguess = a.take<float2>(cf); m.fdye = a.take<float>(cf);
    m.bx = a.take<float2>(cb); m.bv = a.take<float2>(cb); m.bth = a.take<float>(cb); m.bom = a.take<float>(cb);
    m.imp = a.take<float2>(cb); m.ang = a.take<float>(cb);
    m.x0 = a.take<float2>(cf); m.dp = a.take<float2>(cf); m.push_ex = a.take<float2>(cf);
    m.coh_dv = a.take<float2>(cf); m.adh_dv = a.take<float2>(cf); m.dv_tmp = a.take<float2>(cf);
    m.density = a.take<float>(cf); m.lambda = a.take<float>(cf); m.wall_val = a.take<float>(cf);
    m.f_tmp = a.take<float>(cf); m.mu_eff = a.take<float>(cf); m.wall_bin = a.take<int32_t>(cf);
    m.nbr_off = a.take<uint32_t>(cf + 1); m.nbrs = a.take<uint32_t>(m.cap_edges);
    m.visc_w = a.take<float>(m.cap_edges); m.visc_dir = a.take<float2>(m.cap_edges);
    GridBuf* gs[3] = {&m.gA, &m.gB, &m.gBall};
    for (int g = 0; g < 3; ++g) {
      uint32_t pts = g < 2 ? cf : cb, cells = g < 2 ? fcells : bcells;
      gs[g]->cap_points = pts;
      gs[g]->cap_cells = cells;
      gs[g]->pkey = a.take<int2>(pts);
      gs[g]->cell_start = a.take<uint32_t>(cells + 1);
      gs[g]->cursor = a.take<uint32_t>(cells + 1);
      gs[g]->indices = a.take<uint32_t>(pts);
      gs[g]->keys = a.take<int2>(pts);
    }
    m.rec_i = a.take<uint32_t>(m.cap_recs); m.rec_b = a.take<uint32_t>(m.cap_recs);
    m.rec_J = a.take<float2>(m.cap_recs); m.rec_M = a.take<float2>(m.cap_recs);
    m.rec_L = a.take<float>(m.cap_recs);
    m.rec_cnt = a.take<uint32_t>(cf + 1);
    size_t items = (size_t)cb * m.cap_items;
    m.item_j = a.take<uint32_t>(items); m.item_v = a.take<float2>(items);
    m.item_w = a.take<float>(items); m.item_w2 = a.take<float>(items);
    m.item_n = a.take<uint32_t>(cb + 1);
    m.bk_start = a.take<uint32_t>(nbig); m.bk_cur = a.take<uint32_t>(nbig);
    m.bk_order = a.take<uint32_t>(m.cap_recs);
    const size_t nit = (size_t)m.cap_pairs + cb + 1;
    m.dm_pa = a.take<uint32_t>(nit); m.dm_pb = a.take<uint32_t>(nit); m.dm_lvl = a.take<uint32_t>(nit);
    m.lev_start = a.take<uint32_t>(nit + 1); m.lev_cur = a.take<uint32_t>(nit + 1);
    m.lev_items = a.take<uint32_t>(nit);
    m.act_i = a.take<uint32_t>(nit); m.act_j = a.take<uint32_t>(nit); m.act_flag = a.take<uint32_t>(nit + 1);
    m.act_l = a.take<float>(nit); m.act_w1 = a.take<float>(nit); m.act_w2 = a.take<float>(nit);
    m.act_t = a.take<float>(nit);
    m.act_bin = a.take<int32_t>(nit);
    m.act_rec = a.take<MgImpactRecord>(nit);
    m.g_fluid = a.take<uint32_t>(m.cap_groups); m.g_ball = a.take<uint32_t>(m.cap_groups);
    m.g_c = a.take<float>(m.cap_groups); m.g_l2 = a.take<float>(m.cap_groups); m.g_lc = a.take<float2>(m.cap_groups);
    m.g_off = a.take<uint32_t>(cb + 1);
    m.fg_start = a.take<uint32_t>(cf + 1); m.fg_list = a.take<uint32_t>(m.cap_groups);
    m.l_ball = a.take<uint32_t>(m.cap_links); m.l_other = a.take<uint32_t>(m.cap_links);
    m.l_n = a.take<float2>(m.cap_links); m.l_c = a.take<float>(m.cap_links);
    m.l_off = a.take<uint32_t>(cb + 1);
    m.lo_start = a.take<uint32_t>(cb + 2); m.lo_list = a.take<uint32_t>(m.cap_links);
    size_t len = (size_t)cf + 2u * cb;
    m.cg_x = a.take<float2>(len); m.cg_b = a.take<float2>(len); m.cg_r = a.take<float2>(len);
    m.cg_z = a.take<float2>(len); m.cg_p = a.take<float2>(len); m.cg_ap = a.take<float2>(len);
    m.cg_lv = a.take<float2>(cf); m.cg_diag = a.take<float>(len); m.cg_inv = a.take<float>(len);
    m.ball_v0 = a.take<float2>(cb); m.ball_w0 = a.take<float>(cb);
    m.drag_pre = a.take<float>((size_t)8 * cb);
    m.bx0 = a.take<float2>(cb); m.bvpre = a.take<float2>(cb);
    m.bth0 = a.take<float>(cb); m.bompre = a.take<float>(cb); m.lam_bw = a.take<float>(cb);
    m.bxs = a.take<float2>(cb); m.bmove = a.take<float>(cb); m.f_cw = a.take<double>(cb);
    m.rec_off = a.take<uint32_t>(cb + 1); m.rec_pred = a.take<uint32_t>(m.cap_recs);
    m.ball_done = a.take<uint32_t>(cb);
    m.slot = a.take<uint32_t>((size_t)MAX_BLOCK_WARPS * s->mill_blocks_cap * cf);
    if (s->mill_blocks_cap > 1) {
      // the lists and records the helper blocks fill beside the drag sweep
      m.gi_j = a.take<uint32_t>(items); m.gi_v = a.take<float2>(items);
      m.gi_w = a.take<float>(items); m.gi_w2 = a.take<float>(items);
      m.bi_j = a.take<uint32_t>(items); m.bi_v = a.take<float2>(items); m.bi_w = a.take<float>(items);
      m.bi_n = a.take<uint32_t>(cb + 1);
      m.b_rec_off = a.take<uint32_t>(cb + 1); m.b_rec_i = a.take<uint32_t>(items);
      m.b_rec_b = a.take<uint32_t>(items); m.b_rec_pred = a.take<uint32_t>(items);
      m.hb_start = a.take<uint32_t>(nbig); m.hb_cur = a.take<uint32_t>(nbig); m.hb_order = a.take<uint32_t>(items);
      m.b_order = a.take<uint32_t>(cb); m.d_order = a.take<uint32_t>(cb);
      m.lk_j = a.take<uint32_t>(m.cap_links); m.lk_n = a.take<float2>(m.cap_links); m.lk_c = a.take<float>(m.cap_links);
      m.lk_cnt = a.take<uint32_t>(cb); m.lk_winr = a.take<uint32_t>(cb);
      m.lk_wn = a.take<float2>(cb); m.lk_wc = a.take<float>(cb);
    } else {
      m.gi_j = m.bi_j = m.bi_n = m.b_rec_off = m.b_rec_i = m.b_rec_b = m.b_rec_pred = nullptr;
      m.hb_start = m.hb_cur = m.hb_order = m.b_order = m.d_order = nullptr;
      m.lk_j = m.lk_cnt = m.lk_winr = nullptr;
      m.lk_n = m.lk_wn = nullptr;
      m.lk_c = m.lk_wc = nullptr;
      m.gi_v = m.bi_v = nullptr;
      m.gi_w = m.gi_w2 = m.bi_w = nullptr;
    }
    m.wide = a.take<WideCtl>(1);
    s->d_metrics = a.take<MgMetrics>(1);
    m.pair_i = a.take<uint32_t>(m.cap_pairs); m.pair_j = a.take<uint32_t>(m.cap_pairs);
    m.lam_bb = a.take<float>(m.cap_pairs);
    m.pr_list = a.take<uint32_t>(m.cap_pairs);
    m.pair_cnt = a.take<uint32_t>(bcells + 1);
    m.out = a.take<StepOut>(MAX_SUB);
    m.impacts = a.take<MgImpactRecord>((size_t)MAX_SUB * m.cap_impacts);
    if (!pass) {
      s->dbytes = a.off + 256;
      cudaError_t e = s->light ? cudaMallocAsync(&s->dmem, s->dbytes, s->stream) : cudaMalloc(&s->dmem, s->dbytes);
      if (e != cudaSuccess) return fail(s, MG_ERR_CUDA, "cudaMalloc(%zu): %s", s->dbytes, cudaGetErrorString(e));
      cudaMemsetAsync(s->dmem, 0, s->dbytes, s->stream);
    }
  }
  // the merge slot maps are kept all-NONE between uses
  cudaMemsetAsync(m.slot, 0xFF, sizeof(uint32_t) * (size_t)MAX_BLOCK_WARPS * s->mill_blocks_cap * cf, s->stream);
  // the stress accumulator: its state as the handle last saw it, its table re-filled
  CK(cudaMemcpyAsync(m.stress, &s->stress, sizeof(StressState), cudaMemcpyHostToDevice, s->stream));
  if (!old_keys.empty()) {
    std::vector<uint2> keys(m.st_cap, make_uint2(0u, 0u));
    std::vector<double> times(m.st_cap, 0.0);
    const uint32_t mask = m.st_cap - 1u;
    for (size_t q = 0; q < old_keys.size(); ++q) {
      const uint2 k = old_keys[q];
      if (k.x == 0u && k.y == 0u) continue;
      uint32_t slot = stress_slot(k, mask);
      for (uint32_t probe = 0; probe < m.st_cap; ++probe, slot = (slot + 1u) & mask)
        if (keys[slot].x == 0u && keys[slot].y == 0u) { keys[slot] = k; times[slot] = old_times[q]; break; }
    }
    CK(cudaMemcpyAsync(m.st_key, keys.data(), sizeof(uint2) * m.st_cap, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(m.st_time, times.data(), sizeof(double) * m.st_cap, cudaMemcpyHostToDevice, s->stream));
  }
  // the clears must land before anything else touches the arena, whichever stream it uses
  CK(cudaStreamSynchronize(s->stream));
  m.nf = nf;
  m.nb = nb;
  s->md = m;
  s->cap_nf = cf;
  s->cap_nb = cb;
  s->nf = nf;
  s->nb = nb;
  delete[] s->h_imp;
  s->h_imp = new MgImpactRecord[(size_t)MAX_SUB * m.cap_impacts];
  return MG_OK;
}

// The descriptor's per-mill scalars: counts, materials, shared-memory sizing.
void fill_desc(MgSim* s) {
  s->md.nf = s->nf;
  s->md.nb = s->nb;
  s->md.f_mass = s->fmat.particle_mass;
  s->md.f_h = s->fmat.h;
  s->md.f_rho0 = s->fmat.rest_density;
  s->md.b_r = s->bmat.radius;
  s->md.b_m = s->bmat.mass;
  s->md.b_I = s->bmat.inertia;
  s->md.b_rtrue = s->bmat.true_radius;
  s->md.smem_bytes = (uint32_t)stage_smem_bytes(s->nf, s->nb, s->mill_blocks_cap > 1);
  s->md.smem_balls = (size_t)s->nb * 24 <= s->md.smem_bytes ? s->nb : 0u;
  // the mill block's bound on a wait for its helper blocks: ~10 s, or the tests' short limit
  s->md.wide_wait_cycles = s->opt.test_wait_limit_us ? 2000LL * s->opt.test_wait_limit_us : WIDE_TIMEOUT_CYCLES;
  s->md.test_extra_helpers = (s->opt.test_faults & 1u) ? 1u : 0u;
}

int push_desc(MgSim* s) {
  fill_desc(s);
  CK(cudaMemcpyAsync(s->d_md, &s->md, sizeof(MillDev), cudaMemcpyHostToDevice, s->stream));
  return MG_OK;
}

// The sub-step kernel is only launched on materials it is written for: positive, finite fluid
// smoothing length, particle mass and rest density (when there is fluid) and ball radius, mass,
// inertia and true radius (when there are balls).
bool pos_finite(float v) { return v > 0.0f && std::isfinite(v); }
int check_materials(MgSim* s) {
  if (s->nf > 0 && !(pos_finite(s->fmat.h) && pos_finite(s->fmat.particle_mass) && pos_finite(s->fmat.rest_density)))
    return fail(s, MG_ERR_STATE, "fluid material (h, particle mass, rest density) must be positive and finite");
  if (s->nb > 0 && !(pos_finite(s->bmat.radius) && pos_finite(s->bmat.mass) && pos_finite(s->bmat.inertia) &&
                     pos_finite(s->bmat.true_radius)))
    return fail(s, MG_ERR_STATE, "ball material (radius, mass, inertia, true radius) must be positive and finite");
  return MG_OK;
}

// Fills the mill-uniform block for one call (geometry trig, boundary offsets, films).
int fill_uniform(MgSim* s, const MgDrum& drum, const MgMediaParams& media, const MgSlurryParams& slurry,
                 uint32_t pbf_it, uint32_t dem_it, int run_fluid, int run_dem, int ext) {
  StepUniform& U = *s->h_uni;
  std::memset(&U, 0, sizeof(U));
  U.drum_radius = drum.radius_m;
  U.drum_omega = drum.omega;
  if (drum.lifters.count > (uint32_t)MAX_LIFTERS) return fail(s, MG_ERR_ARG, "lifters.count above %d", MAX_LIFTERS);
  U.lifter_count = drum.lifters.count;
  U.lifter_height = drum.lifters.height_m;
  U.lifter_base_half = drum.lifters.base_width_m * 0.5f;
  U.lifter_top_half = drum.lifters.top_width_m * 0.5f;
  const float rads_per_deg = mgh::PI_F / 180.0f;
  float phase = drum.lifters.phase_deg * rads_per_deg;
  for (uint32_t k = 0; k < U.lifter_count; ++k) {
    float th = phase + (float)k * mgh::TAU_F / (float)U.lifter_count;  // geometry.rs:55
    U.lifter_sin[k] = mgh::sinf_r(th);
    U.lifter_cos[k] = mgh::cosf_r(th);
  }
  U.pbf_iterations = pbf_it;
  U.dem_iterations = dem_it;
  U.run_fluid = run_fluid;
  U.run_dem = run_dem;
  U.dem_external = ext;
  U.media = media;
  U.slurry = slurry;
  U.cg_fp64 = s->opt.cg_fp64;
  U.sweep_warps = s->opt.sweep_warps ? s->opt.sweep_warps
                 : s->mill_blocks_cap > 1 ? DEFAULT_SWEEP_WARPS_SINGLE : DEFAULT_SWEEP_WARPS;
  U.spin_ns = s->opt.spin_ns ? s->opt.spin_ns : DEFAULT_SPIN_NS;
  // polls of a waiting ball before it gives up: about a second, or the tests' short limit
  U.spin_limit = s->opt.test_wait_limit_us
                     ? std::max<uint32_t>(1u, (uint32_t)std::min<uint64_t>(
                                                  (uint64_t)s->opt.test_wait_limit_us * 1000u / std::max(U.spin_ns, 1u),
                                                  SPIN_LIMIT))
                     : SPIN_LIMIT;
  U.skip_done_ball = (s->opt.test_faults & 2u) ? 0u : NONE;
  U.sweep_order = s->opt.sweep_order;
  // pbf.rs:190-219: boundary points at dx = h / 2 (adhesion and viscosity groups)
  U.boundary_count = 0;
  float br = s->bmat.radius, dx = 0.5f * s->fmat.h;
  if (s->nb > 0 && s->nf > 0 && br > 0.0f && dx > 0.0f) {
    float circumference = mgh::TAU_F * br;
    uint32_t count = std::max(mgh::f2u_sat(std::round(circumference / dx)), 6u);
    if (count > (uint32_t)MAX_BOUNDARY_POINTS)
      return fail(s, MG_ERR_CAPACITY, "%u boundary points per ball exceed %d", count, MAX_BOUNDARY_POINTS);
    U.boundary_count = count;
    for (uint32_t k = 0; k < count; ++k) {
      float angle = mgh::TAU_F * (float)k / (float)count;
      U.boundary_offset[k] = V2(mgh::cosf_r(angle) * br, mgh::sinf_r(angle) * br);
    }
  }
  // mac/lubrication.rs:49-73 SqueezeFilm::new for the pair (1/a, 1/a) and wall (1/a, -1/b) films
  auto film = [](double k1, double k2, double nu) {
    FilmConsts f;
    f.r = 1.0 / (k1 + k2);
    double q = (f.r * (f.r * f.r)) * (k1 * (k1 * k1) + k2 * (k2 * k2));
    f.c1 = 0.788 + 0.265 * q;
    double c2 = 0.006 + 0.057 * (q - 0.25);
    f.c2 = c2 > 0.0 ? c2 : 0.0;
    f.prefactor = 3.0 * std::sqrt(2.0) * M_PI * nu * std::pow(f.r, 1.5);
    return f;
  };
  double a = (double)br, bd = (double)drum.radius_m, mud = (double)mgh::fmax_r(slurry.viscosity_pa_s, 0.0f);
  if (a > 0.0) {
    U.pair_film = film(1.0 / a, 1.0 / a, mud);
    U.wall_film = film(1.0 / a, -1.0 / bd, mud);
  }
  return MG_OK;
}

// now_s: Simulation::sim_time when the sub-step's impacts are folded (the stress accumulator's
// clock); alpha: the sub-step's EMA weight 1 - exp(-dt / 1 s) in f32 (lib.rs:516-537).
void fill_angle(SubAngles& A, float angle, float omega, float dt, double now_s = 0.0) {
  A.drum_angle = angle;
  A.drum_angle_next = angle + omega * dt;
  A.dt = dt;
  A.pad = 0.0f;
  A.now_s = now_s;
  A.alpha = 1.0f - mgh::expf_r(-dt / 1.0f);
  A.pad2 = 0.0f;
  float an = A.drum_angle_next;
  A.to_local_next = V2(mgh::cosf_r(-an), mgh::sinf_r(-an));
  A.to_world_next = V2(mgh::cosf_r(an), mgh::sinf_r(an));
  A.to_local0 = V2(mgh::cosf_r(-angle), mgh::sinf_r(-angle));
}

// Launches n_sub sub-steps (angles already in h_ang) and waits; outputs land in h_out / h_imp.
int run(MgSim* s, uint32_t n_sub) {
  if (n_sub > MAX_SUB) return fail(s, MG_ERR_ARG, "at most %u sub-steps per launch", MAX_SUB);
  int rc = check_materials(s);
  if (!rc) rc = push_desc(s);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s->d_uni, s->h_uni, sizeof(StepUniform), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->d_ang, s->h_ang, sizeof(SubAngles) * n_sub, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemsetAsync(s->md.err, 0, sizeof(uint32_t), s->stream));
  const uint32_t mill_blocks = s->opt.mill_blocks ? s->opt.mill_blocks : std::min(DEFAULT_MILL_BLOCKS, s->mill_blocks_cap);
  if (mill_blocks > 1) CK(cudaMemsetAsync(s->md.wide, 0, sizeof(WideCtl), s->stream));
  CK(cudaEventRecord(s->ev0, s->stream));
  CK(launch_substeps(s->d_md, 1, s->d_uni, s->d_ang, n_sub, nullptr, s->opt.block_threads, s->md.smem_bytes,
                     s->stream, mill_blocks, nullptr, s->opt.block_regs == 64));
  CK(cudaEventRecord(s->ev1, s->stream));
  CK(cudaMemcpyAsync(s->h_out, s->md.out, sizeof(StepOut) * n_sub, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(&s->stress, s->md.stress, sizeof(StressState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaEventElapsedTime(&s->last_kernel_ms, s->ev0, s->ev1));
  s->launches += 1;
  for (uint32_t k = 0; k < n_sub; ++k) {
    const uint32_t* c = reinterpret_cast<const uint32_t*>(&s->h_out[k].ctr);
    for (int q = 0; q < 10; ++q) s->ctr_tot[q] += c[q];
    for (int q = 0; q < 40; ++q) s->stage_tot[q] += s->h_out[k].stage[q];
    s->ctr_n += 1;
  }
  uint32_t e = 0;
  for (uint32_t k = 0; k < n_sub; ++k) e |= s->h_out[k].err;
  if (e & ERR_WIDE) return fail(s, MG_ERR_CUDA, "the mill's thread blocks stopped waiting for one another (timeout)");
  if (e & ERR_BUDGET)
    return fail(s, MG_ERR_STATE, "a bounded device wait ran out (a ball of a per-ball sweep waited for an earlier "
                                 "ball that never finished; error bits 0x%x)", e);
  if (e) return fail(s, MG_ERR_CAPACITY, "device capacity exceeded (error bits 0x%x)", e);
  size_t total_imp = 0;
  for (uint32_t k = 0; k < n_sub; ++k) total_imp += s->h_out[k].n_impacts;
  if (total_imp) {
    for (uint32_t k = 0; k < n_sub; ++k) {
      uint32_t ni = std::min(s->h_out[k].n_impacts, s->md.cap_impacts);
      if (ni)
        CK(cudaMemcpyAsync(s->h_imp + (size_t)k * s->md.cap_impacts, s->md.impacts + (size_t)k * s->md.cap_impacts,
                           sizeof(MgImpactRecord) * ni, cudaMemcpyDeviceToHost, s->stream));
    }
    CK(cudaStreamSynchronize(s->stream));
  }
  s->last_fluid = s->h_out[n_sub - 1].fs;
  s->last_dem = s->h_out[n_sub - 1].ds;
  s->last_ctr = s->h_out[n_sub - 1].ctr;
  return MG_OK;
}

MgDrum sim_drum(const MgSim* s) {
  MgDrum d;
  d.radius_m = mgh::mill_radius(s->params.mill);
  d.omega = mgh::mill_omega(s->params.mill);
  d.lifters = s->params.lifters;
  return d;
}

// lib.rs:491-565 for sub-step k of the last launch
void fold_substep(MgSim* s, uint32_t k, float sub_dt, float omega) {
  const MgFluidStepStats& fs = s->h_out[k].fs;
  const MgDemStepStats& ds = s->h_out[k].ds;
  s->clamp_hits_frame += fs.coupling_clamp_hits;
  MgEnergyBudget& b = s->budget;
  b.elapsed_s += (double)sub_dt;
  b.dem_wall_work_j += (double)ds.wall_work_j;
  b.fluid_wall_work_j += (double)fs.wall_work_j;
  b.shaft_work_j += (double)(ds.wall_work_j + fs.wall_work_j);
  b.ball_contact_dissipation_j += (double)ds.dissipated_energy_j;
  b.fluid_wall_slip_j += (double)(fs.wall_work_j - fs.ke_delta_noslip_j);
  b.fluid_viscous_j -= (double)fs.ke_delta_viscosity_j;
  b.fluid_clamp_removed_j -= (double)fs.ke_delta_clamp_j;
  b.interface_created_j += (double)(ds.coupling_work_j + fs.ke_delta_drag_j + fs.ke_delta_buoyancy_j);
  b.fluid_wall_angular_impulse += (double)fs.wall_angular_impulse;
  // update_grinding_stats
  float alpha = 1.0f - mgh::expf_r(-sub_dt / 1.0f);
  float p_inst = (ds.wall_work_j + fs.wall_work_j) / sub_dt;
  s->power += alpha * (p_inst - s->power);
  float t_inst = std::fabs(omega) > 1e-6f ? p_inst / omega : 0.0f;
  s->torque += alpha * (t_inst - s->torque);
  // the stress accumulator folded this sub-step's impacts on the device; s->stress holds its
  // state after the launch's last sub-step, which is what the frame reports
  s->collision_rate = (float)stress_total_rate(s->stress);
  float diss = mgh::fmax_r(ds.dissipated_energy_j, 0.0f) / sub_dt;
  s->dissipated_power += alpha * (diss - s->dissipated_power);
  s->max_disp = mgh::fmax_r(s->max_disp, ds.max_substep_displacement_over_diameter);
  s->drum_angle = mgh::rem_euclid_r(s->drum_angle + omega * sub_dt, mgh::TAU_F);
  s->sim_time += (double)sub_dt;
}

// Simulation::step / step_fixed: n sub-steps of sub_dt in one launch, then the bookkeeping.
int advance(MgSim* s, uint32_t n, float sub_dt) {
  MgDrum drum = sim_drum(s);
  float omega = drum.omega;
  const MgSimulationParams& q = s->params.simulation;
  int rc = fill_uniform(s, drum, s->params.media, s->params.slurry, q.pbf_iterations, q.dem_iterations, 1, 1, 1);
  if (rc) return rc;
  s->h_uni->fold_stress = 1u;
  uint32_t done = 0;
  while (done < n) {
    uint32_t chunk = std::min(n - done, MAX_SUB);
    float angle = s->drum_angle;
    double now = s->sim_time;
    for (uint32_t k = 0; k < chunk; ++k) {
      fill_angle(s->h_ang[k], angle, omega, sub_dt, now);
      angle = mgh::rem_euclid_r(angle + omega * sub_dt, mgh::TAU_F);
      now += (double)sub_dt;
    }
    rc = run(s, chunk);
    if (rc) return rc;
    for (uint32_t k = 0; k < chunk; ++k) fold_substep(s, k, sub_dt, omega);
    done += chunk;
  }
  return MG_OK;
}

// A light handle's host blocks (see MgSim::light); it launches nothing of its own.
int init_light_handle(MgSim* s, cudaStream_t stream) {
  s->light = true;
  s->stream = stream;
  s->h_uni = new StepUniform();
  s->h_out = new StepOut[MAX_SUB]();
  return MG_OK;
}

int init_handle(MgSim* s) {
  CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  CK(cudaMalloc(&s->d_md, sizeof(MillDev)));
  CK(cudaMalloc(&s->d_uni, sizeof(StepUniform)));
  CK(cudaMalloc(&s->d_ang, sizeof(SubAngles) * MAX_SUB));
  CK(cudaMallocHost(&s->h_uni, sizeof(StepUniform)));
  CK(cudaMallocHost(&s->h_ang, sizeof(SubAngles) * MAX_SUB));
  CK(cudaMallocHost(&s->h_out, sizeof(StepOut) * MAX_SUB));
  CK(cudaEventCreate(&s->ev0));
  CK(cudaEventCreate(&s->ev1));
  return MG_OK;
}

int upload_balls(MgSim* s, const float* x, const float* v, const float* th, const float* om) {
  size_t n = s->nb;
  if (!n) return MG_OK;
  CK(cudaMemcpyAsync(s->md.bx, x, 8 * n, cudaMemcpyHostToDevice, s->stream));
  if (v) CK(cudaMemcpyAsync(s->md.bv, v, 8 * n, cudaMemcpyHostToDevice, s->stream));
  else CK(cudaMemsetAsync(s->md.bv, 0, 8 * n, s->stream));
  if (th) CK(cudaMemcpyAsync(s->md.bth, th, 4 * n, cudaMemcpyHostToDevice, s->stream));
  else CK(cudaMemsetAsync(s->md.bth, 0, 4 * n, s->stream));
  if (om) CK(cudaMemcpyAsync(s->md.bom, om, 4 * n, cudaMemcpyHostToDevice, s->stream));
  else CK(cudaMemsetAsync(s->md.bom, 0, 4 * n, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MG_OK;
}

int upload_fluid(MgSim* s, const float* x, const float* v, const float* dye, const float* guess) {
  size_t n = s->nf;
  uint32_t gv = guess ? 1u : 0u;
  if (n) {
    CK(cudaMemcpyAsync(s->md.fx, x, 8 * n, cudaMemcpyHostToDevice, s->stream));
    if (v) CK(cudaMemcpyAsync(s->md.fv, v, 8 * n, cudaMemcpyHostToDevice, s->stream));
    else CK(cudaMemsetAsync(s->md.fv, 0, 8 * n, s->stream));
    if (dye) CK(cudaMemcpyAsync(s->md.fdye, dye, 4 * n, cudaMemcpyHostToDevice, s->stream));
    else CK(cudaMemsetAsync(s->md.fdye, 0, 4 * n, s->stream));
    if (guess) CK(cudaMemcpyAsync(s->md.fguess, guess, 8 * n, cudaMemcpyHostToDevice, s->stream));
  }
  CK(cudaMemcpyAsync(s->md.guess_valid_dev, &gv, 4, cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MG_OK;
}

// Simulation::new / with_initial_balls. With a server stream the handle is a light one (MgSim::light).
int create_sim(const MgParams* p, const float* xy, uint32_t n_init, MgSim** out, cudaStream_t server_stream = nullptr,
               uint32_t mill_blocks_cap = 1) {
  if (!p || !out) return fail_global(MG_ERR_ARG, "null argument");
  std::string e;
  if (!mgh::params_validate(*p, &e)) return fail_global(MG_ERR_INVALID_PARAMS, "%s", e.c_str());
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail_global(MG_ERR_NO_DEVICE, "no CUDA device visible");
  MgSim* s = new MgSim();
  s->params = *p;
  s->mill_blocks_cap = std::max<uint32_t>(1u, std::min<uint32_t>(mill_blocks_cap, MAX_MILL_BLOCKS));
  int rc = server_stream ? init_light_handle(s, server_stream) : init_handle(s);
  if (rc) { g_err = s->err; mg_sim_destroy(s); return rc; }
  float radius = mgh::mill_radius(p->mill);
  mgh::Effective eff = mgh::effective_media(*p);
  mgh::Balls balls;
  mgh::seed_balls(&balls, eff, radius, p->simulation.seed);
  if (xy) {
    balls.x.assign(xy, xy + 2 * (size_t)n_init);
    balls.v.assign(2 * (size_t)n_init, 0.0f);
    balls.theta.assign(n_init, 0.0f);
    balls.omega.assign(n_init, 0.0f);
  }
  uint32_t res = mgh::effective_fluid_resolution(*p);
  mgh::Fluid fluid;
  if (p->slurry.enabled) {
    mgh::seed_fluid(&fluid, p->slurry, radius, res, balls.x, balls.radius);
  } else {
    MgSlurryParams sp = p->slurry;
    sp.fill_fraction = 0.0f;
    mgh::seed_fluid(&fluid, sp, radius, res, std::vector<float>(), 0.0f);
  }
  if (xy) {
    float w = mgh::mill_omega(p->mill);
    for (size_t i = 0; i < balls.len(); ++i) {
      balls.v[2 * i] = w * -balls.x[2 * i + 1];
      balls.v[2 * i + 1] = w * balls.x[2 * i];
      balls.omega[i] = w;
    }
    for (size_t i = 0; i < fluid.len(); ++i) {
      fluid.v[2 * i] = w * -fluid.x[2 * i + 1];
      fluid.v[2 * i + 1] = w * fluid.x[2 * i];
    }
  }
  s->bmat = {balls.radius, balls.mass, balls.inertia, balls.true_radius};
  s->fmat = {fluid.particle_mass, fluid.h, fluid.rest_density};
  s->e0 = mgh::balls_energy_f64(balls) + mgh::fluid_energy_f64(fluid);
  rc = alloc_state(s, (uint32_t)fluid.len(), (uint32_t)balls.len());
  if (!rc) rc = upload_balls(s, balls.x.data(), balls.v.data(), balls.theta.data(), balls.omega.data());
  if (!rc) rc = upload_fluid(s, fluid.x.data(), fluid.v.data(), fluid.dye.data(), nullptr);
  if (rc) { g_err = s->err; mg_sim_destroy(s); return rc; }
  *out = s;
  return MG_OK;
}

int download(MgSim* s, mgh::Balls* b, mgh::Fluid* f) {
  if (b) {
    b->x.resize(2 * s->nb); b->v.resize(2 * s->nb); b->theta.resize(s->nb); b->omega.resize(s->nb);
    if (s->nb) {
      CK(cudaMemcpyAsync(b->x.data(), s->md.bx, 8 * s->nb, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaMemcpyAsync(b->v.data(), s->md.bv, 8 * s->nb, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaMemcpyAsync(b->theta.data(), s->md.bth, 4 * s->nb, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaMemcpyAsync(b->omega.data(), s->md.bom, 4 * s->nb, cudaMemcpyDeviceToHost, s->stream));
    }
    b->radius = s->bmat.radius; b->mass = s->bmat.mass; b->inertia = s->bmat.inertia; b->true_radius = s->bmat.true_radius;
  }
  if (f) {
    f->x.resize(2 * s->nf); f->v.resize(2 * s->nf); f->dye.resize(s->nf);
    if (s->nf) {
      CK(cudaMemcpyAsync(f->x.data(), s->md.fx, 8 * s->nf, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaMemcpyAsync(f->v.data(), s->md.fv, 8 * s->nf, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaMemcpyAsync(f->dye.data(), s->md.fdye, 4 * s->nf, cudaMemcpyDeviceToHost, s->stream));
    }
    f->particle_mass = s->fmat.particle_mass; f->h = s->fmat.h; f->rest_density = s->fmat.rest_density;
  }
  CK(cudaStreamSynchronize(s->stream));
  return MG_OK;
}

}  // namespace

namespace mg {
int set_global_error(int code, const char* msg) { return fail_global(code, "%s", msg); }
}  // namespace mg

// ====================================================================== C ABI
extern "C" {

size_t mg_sizeof_params(void) { return sizeof(MgParams); }
size_t mg_sizeof_fluid_stats(void) { return sizeof(MgFluidStepStats); }
size_t mg_sizeof_dem_stats(void) { return sizeof(MgDemStepStats); }

int mg_params_default(MgParams* out) {
  if (!out) return fail_global(MG_ERR_ARG, "null argument");
  *out = mgh::params_default();
  return MG_OK;
}
int mg_params_validate(const MgParams* p, char* err, size_t n) {
  if (!p) return fail_global(MG_ERR_ARG, "null argument");
  std::string e;
  if (mgh::params_validate(*p, &e)) return MG_OK;
  if (err && n) { std::strncpy(err, e.c_str(), n - 1); err[n - 1] = 0; }
  return fail_global(MG_ERR_INVALID_PARAMS, "%s", e.c_str());
}
int mg_preset_apply(MgParams* p, const char* id) {
  if (!p) return fail_global(MG_ERR_ARG, "null argument");
  return mgh::preset_apply(p, id) ? MG_OK : fail_global(MG_ERR_ARG, "unknown preset '%s'", id ? id : "");
}
int mg_params_derived(const MgParams* pp, MgDerived* o) {
  if (!pp || !o) return fail_global(MG_ERR_ARG, "null argument");
  const MgParams& p = *pp;
  mgh::Effective e = mgh::effective_media(p);
  o->critical_speed_rpm = mgh::critical_speed_rpm(p.mill);
  o->rpm = mgh::mill_rpm(p.mill);
  o->percent_critical = mgh::mill_percent_critical(p.mill);
  o->omega = mgh::mill_omega(p.mill);
  o->radius_m = mgh::mill_radius(p.mill);
  o->true_ball_count = mgh::true_ball_count(p);
  o->eff_true_diameter_m = e.true_diameter_m;
  o->eff_diameter_m = e.diameter_m;
  o->eff_density_kg_m3 = e.density_kg_m3;
  o->eff_ball_count = e.ball_count;
  o->eff_scale_factor = e.scale_factor;
  o->effective_fluid_resolution = mgh::effective_fluid_resolution(p);
  o->effective_substeps = mgh::effective_substeps(p);
  o->fixed_sub_dt = 1.0f / (60.0f * (float)std::max(o->effective_substeps, 1u));
  return MG_OK;
}

int mg_sim_create(const MgParams* p, MgSim** out) { return create_sim(p, nullptr, 0, out, nullptr, MAX_MILL_BLOCKS); }
int mg_sim_create_with_balls(const MgParams* p, const float* xy, uint32_t n, MgSim** out) {
  if (!xy && n) return fail_global(MG_ERR_ARG, "null positions");
  static const float dummy[2] = {0.0f, 0.0f};
  return create_sim(p, xy ? xy : dummy, n, out, nullptr, MAX_MILL_BLOCKS);
}
void mg_sim_destroy(MgSim* s) {
  if (!s) return;
  if (s->light) {
    // the arena goes back to the pool in stream order; the stream belongs to the server
    if (s->dmem) cudaFreeAsync(s->dmem, s->stream);
    if (s->surf_mem) cudaFreeAsync(s->surf_mem, s->stream);
    if (s->h_surf) {
      cudaStreamSynchronize(s->stream);
      cudaFreeHost(s->h_surf);
    }
    delete s->h_uni;
    delete[] s->h_out;
    delete[] s->h_imp;
    delete s;
    return;
  }
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->dmem) cudaFree(s->dmem);
  if (s->surf_mem) cudaFree(s->surf_mem);
  if (s->h_surf) cudaFreeHost(s->h_surf);
  if (s->d_md) cudaFree(s->d_md);
  if (s->d_uni) cudaFree(s->d_uni);
  if (s->d_ang) cudaFree(s->d_ang);
  if (s->h_uni) cudaFreeHost(s->h_uni);
  if (s->h_ang) cudaFreeHost(s->h_ang);
  if (s->h_out) cudaFreeHost(s->h_out);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete[] s->h_imp;
  delete s;
}
const char* mg_last_error(const MgSim* s) { return s ? s->err.c_str() : g_err.c_str(); }
const char* mg_global_last_error(void) { return g_err.c_str(); }
int mg_sim_set_options(MgSim* s, const MgOptions* o) {
  if (!s || !o) return fail(s, MG_ERR_ARG, "null argument");
  if (o->block_threads != 0 && (o->block_threads % 32 != 0 || o->block_threads > MAX_BLOCK_THREADS))
    return fail(s, MG_ERR_ARG, "block_threads must be a multiple of 32 in [32, %u]", MAX_BLOCK_THREADS);
  if (o->sweep_warps > MAX_BLOCK_WARPS) return fail(s, MG_ERR_ARG, "sweep_warps must be in [0, %u]", MAX_BLOCK_WARPS);
  if (o->spin_ns > 100000) return fail(s, MG_ERR_ARG, "spin_ns must be at most 100000");
  if (o->mill_blocks > s->mill_blocks_cap)
    return fail(s, MG_ERR_ARG, "mill_blocks must be in [0, %u] for this handle", s->mill_blocks_cap);
  if (o->test_wait_limit_us > 10000000u) return fail(s, MG_ERR_ARG, "test_wait_limit_us must be at most 10000000");
  if (o->test_faults & ~3u) return fail(s, MG_ERR_ARG, "test_faults: only bits 1 and 2 are defined");
  if (o->block_regs != 0 && o->block_regs != 64) return fail(s, MG_ERR_ARG, "block_regs must be 0 or 64");
  if (o->sweep_order > 1) return fail(s, MG_ERR_ARG, "sweep_order must be 0 (by level) or 1 (index order)");
  s->opt = *o;
  return MG_OK;
}
int mg_sim_step(MgSim* s, float dt) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  uint32_t n = std::max(mgh::effective_substeps(s->params), 1u);
  float sub_dt = dt / (float)n;
  s->max_disp = 0.0f;
  s->clamp_hits_frame = 0;
  return advance(s, n, sub_dt);
}
int mg_sim_step_fixed(MgSim* s) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  return advance(s, 1, mg_sim_fixed_sub_dt(s));
}
int mg_sim_reset_frame_stats(MgSim* s) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  s->max_disp = 0.0f;
  s->clamp_hits_frame = 0;
  return MG_OK;
}
int mg_sim_set_params(MgSim* s, const MgParams* p) {
  if (!s || !p) return fail(s, MG_ERR_ARG, "null argument");
  std::string e;
  if (!mgh::params_validate(*p, &e)) return fail(s, MG_ERR_INVALID_PARAMS, "%s", e.c_str());
  s->params = *p;
  return MG_OK;
}
float mg_sim_fixed_sub_dt(const MgSim* s) {
  return 1.0f / (60.0f * (float)std::max(mgh::effective_substeps(s->params), 1u));
}
int mg_sim_reset_energy_budget(MgSim* s) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  mgh::Balls b;
  mgh::Fluid f;
  int rc = download(s, &b, &f);
  if (rc) return rc;
  std::memset(&s->budget, 0, sizeof(s->budget));
  s->e0 = mgh::balls_energy_f64(b) + mgh::fluid_energy_f64(f);
  return MG_OK;
}

int mg_coupling_step_recorded(MgSim* s, const MgDrum* drum, float drum_angle, const MgMediaParams* media,
                              const MgSlurryParams* slurry, uint32_t dem_it, uint32_t pbf_it, float dt,
                              MgFluidStepStats* fstats, MgDemStepStats* dstats, MgImpactRecord* out, uint32_t cap,
                              uint32_t* n_out) {
  if (!s || !drum || !media || !slurry) return fail(s, MG_ERR_ARG, "null argument");
  int rc = fill_uniform(s, *drum, *media, *slurry, pbf_it, dem_it, 1, 1, 1);
  if (rc) return rc;
  fill_angle(s->h_ang[0], drum_angle, drum->omega, dt);
  rc = run(s, 1);
  if (rc) return rc;
  if (fstats) *fstats = s->h_out[0].fs;
  if (dstats) *dstats = s->h_out[0].ds;
  uint32_t ni = std::min(s->h_out[0].n_impacts, s->md.cap_impacts);
  if (n_out) *n_out = s->h_out[0].n_impacts;
  if (out) std::memcpy(out, s->h_imp, sizeof(MgImpactRecord) * std::min(ni, cap));
  return MG_OK;
}

int mg_fluid_step_coupled(MgSim* s, const MgDrum* drum, float drum_angle, const MgSlurryParams* slurry,
                          uint32_t it, float dt, MgFluidStepStats* fstats, float* impulses, float* angular,
                          uint32_t* clamp_hits, float* fluid_momentum) {
  if (!s || !drum || !slurry) return fail(s, MG_ERR_ARG, "null argument");
  int rc = fill_uniform(s, *drum, s->params.media, *slurry, it, 1, 1, 0, 1);
  if (rc) return rc;
  s->h_uni->want_momentum = 1;  // CouplingImpulses::fluid_momentum_change is returned here only
  fill_angle(s->h_ang[0], drum_angle, drum->omega, dt);
  rc = run(s, 1);
  if (rc) return rc;
  if (fstats) *fstats = s->h_out[0].fs;
  if (clamp_hits) *clamp_hits = s->h_out[0].clamp_hits;
  if (fluid_momentum) { fluid_momentum[0] = s->h_out[0].fluid_momentum[0]; fluid_momentum[1] = s->h_out[0].fluid_momentum[1]; }
  if (s->nb) {
    if (impulses) CK(cudaMemcpyAsync(impulses, s->md.imp, 8 * s->nb, cudaMemcpyDeviceToHost, s->stream));
    if (angular) CK(cudaMemcpyAsync(angular, s->md.ang, 4 * s->nb, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return MG_OK;
}

int mg_dem_step_recorded(MgSim* s, const MgDrum* drum, float drum_angle, const MgMediaParams* media, uint32_t it,
                         float dt, const float* impulses, const float* angular, MgDemStepStats* dstats,
                         MgImpactRecord* out, uint32_t cap, uint32_t* n_out) {
  if (!s || !drum || !media) return fail(s, MG_ERR_ARG, "null argument");
  int ext = (impulses || angular) ? 1 : 0;
  int rc = fill_uniform(s, *drum, *media, s->params.slurry, 1, it, 0, 1, ext);
  if (rc) return rc;
  if (s->nb) {
    if (impulses) CK(cudaMemcpyAsync(s->md.imp, impulses, 8 * s->nb, cudaMemcpyHostToDevice, s->stream));
    else CK(cudaMemsetAsync(s->md.imp, 0, 8 * s->nb, s->stream));
    if (angular) CK(cudaMemcpyAsync(s->md.ang, angular, 4 * s->nb, cudaMemcpyHostToDevice, s->stream));
    else CK(cudaMemsetAsync(s->md.ang, 0, 4 * s->nb, s->stream));
  }
  fill_angle(s->h_ang[0], drum_angle, drum->omega, dt);
  rc = run(s, 1);
  if (rc) return rc;
  if (dstats) *dstats = s->h_out[0].ds;
  uint32_t ni = std::min(s->h_out[0].n_impacts, s->md.cap_impacts);
  if (n_out) *n_out = s->h_out[0].n_impacts;
  if (out) std::memcpy(out, s->h_imp, sizeof(MgImpactRecord) * std::min(ni, cap));
  return MG_OK;
}

int mg_get_counts(const MgSim* s, uint32_t* nb, uint32_t* nf) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  if (nb) *nb = s->nb;
  if (nf) *nf = s->nf;
  return MG_OK;
}
int mg_get_balls(MgSim* s, float* x, float* v, float* theta, float* omega) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  size_t n = s->nb;
  if (!n) return MG_OK;
  if (x) CK(cudaMemcpyAsync(x, s->md.bx, 8 * n, cudaMemcpyDeviceToHost, s->stream));
  if (v) CK(cudaMemcpyAsync(v, s->md.bv, 8 * n, cudaMemcpyDeviceToHost, s->stream));
  if (theta) CK(cudaMemcpyAsync(theta, s->md.bth, 4 * n, cudaMemcpyDeviceToHost, s->stream));
  if (omega) CK(cudaMemcpyAsync(omega, s->md.bom, 4 * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MG_OK;
}
int mg_set_balls(MgSim* s, uint32_t n, const float* x, const float* v, const float* theta, const float* omega) {
  if (!s || (!x && n)) return fail(s, MG_ERR_ARG, "null argument");
  if (n > s->cap_nb) {
    // grow: keep the fluid state across the reallocation
    mgh::Fluid f;
    int rc = download(s, nullptr, &f);
    std::vector<float> guess(2 * (size_t)s->nf);
    uint32_t gv = 0;
    if (!rc && s->nf) {
      CK(cudaMemcpyAsync(guess.data(), s->md.fguess, 8 * (size_t)s->nf, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaMemcpyAsync(&gv, s->md.guess_valid_dev, 4, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
    }
    uint32_t nf = s->nf;
    if (!rc) rc = alloc_state(s, nf, n);
    if (!rc) rc = upload_fluid(s, f.x.data(), f.v.data(), f.dye.data(), gv ? guess.data() : nullptr);
    if (rc) return rc;
  }
  s->nb = n;
  s->md.nb = n;
  return upload_balls(s, x, v, theta, omega);
}
int mg_get_ball_material(const MgSim* s, MgBallMaterial* o) {
  if (!s || !o) return fail_global(MG_ERR_ARG, "null argument");
  *o = s->bmat;
  return MG_OK;
}
int mg_set_ball_material(MgSim* s, const MgBallMaterial* m) {
  if (!s || !m) return fail(s, MG_ERR_ARG, "null argument");
  s->bmat = *m;
  return MG_OK;
}
int mg_get_fluid(MgSim* s, float* x, float* v, float* dye, float* guess, uint32_t* guess_len) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  size_t n = s->nf;
  uint32_t gv = 0;
  CK(cudaMemcpyAsync(&gv, s->md.guess_valid_dev, 4, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (guess_len) *guess_len = gv ? (uint32_t)n : 0u;
  if (!n) return MG_OK;
  if (x) CK(cudaMemcpyAsync(x, s->md.fx, 8 * n, cudaMemcpyDeviceToHost, s->stream));
  if (v) CK(cudaMemcpyAsync(v, s->md.fv, 8 * n, cudaMemcpyDeviceToHost, s->stream));
  if (dye) CK(cudaMemcpyAsync(dye, s->md.fdye, 4 * n, cudaMemcpyDeviceToHost, s->stream));
  if (guess && gv) CK(cudaMemcpyAsync(guess, s->md.fguess, 8 * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MG_OK;
}
int mg_set_fluid(MgSim* s, uint32_t n, const float* x, const float* v, const float* dye, const float* guess) {
  if (!s || (!x && n)) return fail(s, MG_ERR_ARG, "null argument");
  if (n > s->cap_nf) {
    mgh::Balls b;
    int rc = download(s, &b, nullptr);
    uint32_t nb = s->nb;
    if (!rc) rc = alloc_state(s, n, nb);
    if (!rc) rc = upload_balls(s, b.x.data(), b.v.data(), b.theta.data(), b.omega.data());
    if (rc) return rc;
  }
  s->nf = n;
  s->md.nf = n;
  return upload_fluid(s, x, v, dye, guess);
}
int mg_get_fluid_material(const MgSim* s, MgFluidMaterial* o) {
  if (!s || !o) return fail_global(MG_ERR_ARG, "null argument");
  *o = s->fmat;
  return MG_OK;
}
int mg_set_fluid_material(MgSim* s, const MgFluidMaterial* m) {
  if (!s || !m) return fail(s, MG_ERR_ARG, "null argument");
  s->fmat = *m;
  return MG_OK;
}

int mg_get_scalars(MgSim* s, MgScalars* o) {
  if (!s || !o) return fail_global(MG_ERR_ARG, "null argument");
  std::memset(o, 0, sizeof(*o));
  o->drum_angle = s->drum_angle;
  o->power_draw_w = s->power;
  o->torque_nm = s->torque;
  o->collision_rate_per_s = s->collision_rate;
  o->dissipated_power_w = s->dissipated_power;
  o->max_substep_displacement_over_diameter = s->max_disp;
  o->coupling_clamp_hits = s->clamp_hits_frame;
  o->viscosity_iterations = s->last_fluid.viscosity_iterations;
  o->mean_shear_rate_per_s = s->last_fluid.mean_shear_rate_per_s;
  o->sim_time = s->sim_time;
  return MG_OK;
}
int mg_energy_budget(MgSim* s, MgEnergyBudget* o) {
  if (!s || !o) return fail_global(MG_ERR_ARG, "null argument");
  mgh::Balls b;
  mgh::Fluid f;
  int rc = download(s, &b, &f);
  if (rc) return rc;
  MgEnergyBudget e = s->budget;
  e.delta_mechanical_j = mgh::balls_energy_f64(b) + mgh::fluid_energy_f64(f) - s->e0;
  double explained = e.shaft_work_j - e.ball_contact_dissipation_j - e.fluid_wall_slip_j - e.fluid_viscous_j -
                     e.fluid_clamp_removed_j + e.interface_created_j;
  e.unattributed_j = e.delta_mechanical_j - explained;
  *o = e;
  return MG_OK;
}
int mg_state_hash(MgSim* s, int extended, uint64_t* out) {
  if (!s || !out) return fail_global(MG_ERR_ARG, "null argument");
  mgh::Balls b;
  mgh::Fluid f;
  int rc = download(s, &b, &f);
  if (rc) return rc;
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](float v) {
    uint32_t bits;
    std::memcpy(&bits, &v, 4);
    for (int k = 0; k < 4; ++k) { h ^= (uint64_t)((bits >> (8 * k)) & 0xFFu); h *= 0x100000001b3ull; }
  };
  for (size_t i = 0; i < b.len(); ++i) {
    mix(b.x[2 * i]); mix(b.x[2 * i + 1]); mix(b.v[2 * i]); mix(b.v[2 * i + 1]); mix(b.omega[i]);
    if (extended) mix(b.theta[i]);
  }
  for (size_t i = 0; i < f.len(); ++i) {
    mix(f.x[2 * i]); mix(f.x[2 * i + 1]); mix(f.v[2 * i]); mix(f.v[2 * i + 1]);
    if (extended) mix(f.dye[i]);
  }
  *out = h;
  return MG_OK;
}
int mg_mixing_index(MgSim* s, float* out, int* valid) {
  if (!s || !out || !valid) return fail_global(MG_ERR_ARG, "null argument");
  mgh::Fluid f;
  int rc = download(s, nullptr, &f);
  if (rc) return rc;
  // metrics.rs:506-576 (16 x 16 dye grid, count-weighted Lacey index)
  const int G = 16;
  *valid = 0;
  *out = 0.0f;
  size_t n = f.len();
  float r = mgh::mill_radius(s->params.mill);
  if (n == 0 || r <= 0.0f) return MG_OK;
  float cell = 2.0f * r / (float)G;
  float dye_sum[G * G] = {};
  uint32_t count[G * G] = {};
  float total = 0.0f;
  for (size_t i = 0; i < n; ++i) {
    int32_t gi = std::min(std::max(mgh::f2i_sat(std::floor((f.x[2 * i] + r) / cell)), 0), G - 1);
    int32_t gj = std::min(std::max(mgh::f2i_sat(std::floor((f.x[2 * i + 1] + r) / cell)), 0), G - 1);
    dye_sum[gj * G + gi] += f.dye[i];
    count[gj * G + gi] += 1;
    total += f.dye[i];
  }
  float p_mean = total / (float)n;
  std::vector<float> means;
  std::vector<uint32_t> counts;
  for (int k = 0; k < G * G; ++k)
    if (count[k]) { means.push_back(dye_sum[k] / (float)count[k]); counts.push_back(count[k]); }
  if (means.size() < 2) return MG_OK;
  uint32_t ws = 0;
  for (uint32_t c : counts) ws += c;
  float wsum = (float)ws, ov = 0.0f, wa = 0.0f;
  for (size_t q = 0; q < means.size(); ++q) { float dm = means[q] - p_mean; ov += (float)counts[q] * (dm * dm); }
  float observed = ov / wsum;
  float s0 = p_mean * (1.0f - p_mean);
  for (uint32_t c : counts) wa += (float)c * (float)c;
  float sr = s0 / mgh::fmax_r(wa / wsum, 1.0f);
  if (s0 < 1e-9f) return MG_OK;
  float denom = s0 - sr;
  *valid = 1;
  if (std::fabs(denom) < 1e-9f) { *out = 1.0f; return MG_OK; }
  *out = mgh::clamp_r((s0 - observed) / denom, 0.0f, 1.0f);
  return MG_OK;
}
// metrics::compute (metrics.rs:195-273) on the device, for the current drum angle
// Uploads the uniform of the handle's current state (drum at s->drum_angle, rotations
// from_angle(-angle) and from_angle(angle)) for the launches that read the state in place.
static int push_state_uniform(MgSim* s) {
  MgDrum drum = sim_drum(s);
  int rc = fill_uniform(s, drum, s->params.media, s->params.slurry, 1, 1, 1, 1, 0);
  if (rc) return rc;
  StepUniform& U = *s->h_uni;
  const float a = s->drum_angle;
  U.drum_angle = U.drum_angle_next = a;
  U.to_local_next = V2(mgh::cosf_r(-a), mgh::sinf_r(-a));  // Vec2::from_angle(-angle)
  U.to_world_next = V2(mgh::cosf_r(a), mgh::sinf_r(a));
  U.to_local0 = U.to_local_next;
  rc = check_materials(s);
  if (!rc) rc = push_desc(s);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s->d_uni, s->h_uni, sizeof(StepUniform), cudaMemcpyHostToDevice, s->stream));
  return MG_OK;
}

int mg_metrics(MgSim* s, MgMetrics* out) {
  if (!s || !out) return fail_global(MG_ERR_ARG, "null argument");
  int rc = push_state_uniform(s);
  if (rc) return rc;
  CK(cudaMemsetAsync(s->md.err, 0, sizeof(uint32_t), s->stream));
  CK(launch_metrics(s->d_md, s->d_uni, s->d_metrics, s->stream));
  uint32_t e = 0;
  CK(cudaMemcpyAsync(out, s->d_metrics, sizeof(MgMetrics), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(&e, s->md.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (e) return fail(s, MG_ERR_CAPACITY, "device capacity exceeded in the metrics (error bits 0x%x)", e);
  return MG_OK;
}
// The free-surface scratch, allocated on first use: field, chains, polygon records, output and
// header in one block.
constexpr uint32_t SURF_STAGE = 16384;
static int surf_scratch(MgSim* s) {
  if (s->surf_mem) return MG_OK;
  const size_t n_field = (size_t)SURF_G * SURF_G;
  const size_t bytes = 4 * (n_field + 2 * (size_t)SURF_MAX_SEGS + SURF_WALK_CAP + 3 * (size_t)SURF_MAX_SEGS +
                            SURF_OUT_CAP + 4);
  cudaError_t e = s->light ? cudaMallocAsync(&s->surf_mem, bytes, s->stream) : cudaMalloc(&s->surf_mem, bytes);
  if (e != cudaSuccess) {
    s->surf_mem = nullptr;
    return fail(s, MG_ERR_CUDA, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  float* f = (float*)s->surf_mem;
  SurfDev& sd = s->surf;
  sd.field = f;
  sd.segs = (uint32_t*)(f + n_field);
  sd.walk = sd.segs + 2 * (size_t)SURF_MAX_SEGS;
  sd.poly = sd.walk + SURF_WALK_CAP;
  sd.hdr = sd.poly + 3 * (size_t)SURF_MAX_SEGS;  // the output follows the header, so that one
  sd.phi_full = (float*)(sd.hdr + 2);            // copy brings back both when the surface is small
  sd.out = (float*)(sd.hdr + 4);
  e = cudaMallocHost(&s->h_surf, sizeof(uint32_t) * (4 + SURF_STAGE));
  if (e != cudaSuccess) {
    s->h_surf = nullptr;
    return fail(s, MG_ERR_CUDA, "cudaMallocHost: %s", cudaGetErrorString(e));
  }
  return MG_OK;
}

int mg_fluid_surface(MgSim* s, float* out, uint32_t cap, uint32_t* len) {
  if (!s || !len) return fail_global(MG_ERR_ARG, "null argument");
  int rc = surf_scratch(s);
  if (!rc) rc = push_state_uniform(s);
  if (rc) return rc;
  CK(launch_surface(s->d_md, s->d_uni, s->surf, true, s->stream));
  // header and the first SURF_STAGE floats in one copy; the rest, if any, in a second
  const uint32_t first = out ? std::min<uint32_t>(cap, SURF_STAGE) : 0u;
  CK(cudaMemcpyAsync(s->h_surf, s->surf.hdr, sizeof(uint32_t) * (4 + first), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const uint32_t n = s->h_surf[0];
  *len = n;
  if (!out) return MG_OK;
  if (cap < n) return fail(s, MG_ERR_CAPACITY, "surface needs %u floats, buffer holds %u", n, cap);
  std::memcpy(out, s->h_surf + 4, sizeof(float) * std::min(n, first));
  if (n > first) {
    CK(cudaMemcpyAsync(out + first, s->surf.out + first, sizeof(float) * (n - first), cudaMemcpyDeviceToHost,
                       s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return MG_OK;
}

int mg_surface_field(MgSim* s, float* field, float* phi_full) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  int rc = surf_scratch(s);
  if (!rc) rc = push_state_uniform(s);
  if (rc) return rc;
  CK(launch_surface(s->d_md, s->d_uni, s->surf, false, s->stream));
  if (field)
    CK(cudaMemcpyAsync(field, s->surf.field, sizeof(float) * SURF_G * SURF_G, cudaMemcpyDeviceToHost, s->stream));
  if (phi_full) CK(cudaMemcpyAsync(phi_full, s->surf.phi_full, sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MG_OK;
}

int mg_fluid_densities(MgSim* s, float* out) {
  if (!s || !out) return fail_global(MG_ERR_ARG, "null argument");
  // the metrics launch computes FluidParticles::densities into the sub-step scratch
  int rc = push_state_uniform(s);
  if (rc) return rc;
  CK(cudaMemsetAsync(s->md.err, 0, sizeof(uint32_t), s->stream));
  CK(launch_metrics(s->d_md, s->d_uni, s->d_metrics, s->stream));
  uint32_t e = 0;
  if (s->nf) CK(cudaMemcpyAsync(out, s->md.f_tmp, sizeof(float) * s->nf, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(&e, s->md.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (e) return fail(s, MG_ERR_CAPACITY, "device capacity exceeded computing the densities (error bits 0x%x)", e);
  return MG_OK;
}
int mg_stress_histogram_rate(MgSim* s, double* out28) {
  if (!s || !out28) return fail_global(MG_ERR_ARG, "null argument");
  std::memcpy(out28, s->stress.hist_rate, sizeof(double) * MG_SE_BINS);  // the device state after the last launch
  return MG_OK;
}
int mg_last_step_stats(MgSim* s, MgFluidStepStats* f, MgDemStepStats* d, MgStepCounters* c) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  if (f) *f = s->last_fluid;
  if (d) *d = s->last_dem;
  if (c) *c = s->last_ctr;
  return MG_OK;
}

int mg_sim_stream(MgSim* s, void** stream) {
  if (!s || !stream) return fail_global(MG_ERR_ARG, "null argument");
  *stream = (void*)s->stream;
  return MG_OK;
}
int mg_sim_last_kernel_ms(MgSim* s, float* ms, uint64_t* launches) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  if (ms) *ms = s->last_kernel_ms;
  if (launches) *launches = s->launches;
  return MG_OK;
}
int mg_counter_totals(MgSim* s, uint64_t* totals10, uint64_t* n_substeps, int reset) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  if (totals10) std::memcpy(totals10, s->ctr_tot, sizeof(s->ctr_tot));
  if (n_substeps) *n_substeps = s->ctr_n;
  if (reset) { std::memset(s->ctr_tot, 0, sizeof(s->ctr_tot)); s->ctr_n = 0; }
  return MG_OK;
}

int mg_stage_cycles(MgSim* s, uint64_t* cycles40, int reset) {
  if (!s) return fail_global(MG_ERR_ARG, "null handle");
  if (cycles40) std::memcpy(cycles40, s->stage_tot, sizeof(s->stage_tot));
  if (reset) std::memset(s->stage_tot, 0, sizeof(s->stage_tot));
  return MG_OK;
}

int mg_last_neighbor_lists(MgSim* s, uint32_t* offsets, uint32_t* nbrs, uint32_t cap, uint32_t* n_edges) {
  if (!s || !offsets || !n_edges) return fail_global(MG_ERR_ARG, "null argument");
  CK(cudaMemcpy(offsets, s->md.nbr_off, 4 * ((size_t)s->nf + 1), cudaMemcpyDeviceToHost));
  uint32_t ne = s->nf ? offsets[s->nf] : 0;
  *n_edges = ne;
  if (ne > cap) return fail(s, MG_ERR_CAPACITY, "neighbour buffer too small");
  if (ne && nbrs) CK(cudaMemcpy(nbrs, s->md.nbrs, 4 * (size_t)ne, cudaMemcpyDeviceToHost));
  return MG_OK;
}
int mg_last_ball_pairs(MgSim* s, uint32_t* pairs, uint32_t cap, uint32_t* n_out) {
  if (!s || !n_out) return fail_global(MG_ERR_ARG, "null argument");
  uint32_t np = s->last_ctr.n_ball_pairs;
  *n_out = np;
  if (np > cap) return fail(s, MG_ERR_CAPACITY, "pair buffer too small");
  std::vector<uint32_t> pi(np), pj(np);
  if (np) {
    CK(cudaMemcpy(pi.data(), s->md.pair_i, 4 * (size_t)np, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(pj.data(), s->md.pair_j, 4 * (size_t)np, cudaMemcpyDeviceToHost));
  }
  for (uint32_t k = 0; k < np; ++k) { pairs[2 * k] = pi[k]; pairs[2 * k + 1] = pj[k]; }
  return MG_OK;
}

// ---- grid-stage probes: a scratch mill holding only the caller's points
static int probe(const float* xy, uint32_t n, float cell, int mode, MgSim** out_s, uint32_t res[9]) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail_global(MG_ERR_NO_DEVICE, "no CUDA device visible");
  if (!(cell > 0.0f) || !std::isfinite(cell)) return fail_global(MG_ERR_ARG, "cell_size must be positive");
  MgSim* s = new MgSim();
  s->params = mgh::params_default();
  int rc = init_handle(s);
  // the probe grid lives in the fluid-side buffers; the pair buffers are sized by the ball count
  if (!rc) rc = alloc_state(s, n, std::max(n, 1u));
  if (!rc && n) {
    cudaError_t e = cudaMemcpyAsync(s->md.fx, xy, 8 * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) rc = fail(s, MG_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  s->nb = 0;
  if (!rc) rc = push_desc(s);
  uint32_t* d_res = nullptr;
  if (!rc && cudaMalloc(&d_res, 9 * sizeof(uint32_t)) != cudaSuccess) rc = fail(s, MG_ERR_CUDA, "cudaMalloc");
  if (!rc) {
    cudaMemsetAsync(s->md.err, 0, 4, s->stream);
    cudaError_t e = launch_probe(s->d_md, cell, mode, d_res, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(res, d_res, 9 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) rc = fail(s, MG_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  if (d_res) cudaFree(d_res);
  if (rc) { g_err = s->err; mg_sim_destroy(s); return rc; }
  *out_s = s;
  return MG_OK;
}

int mg_probe_grid(const float* xy, uint32_t n, float cell, int32_t* min_cxy, int64_t* wh, uint32_t* cell_start,
                  uint32_t cell_cap, uint32_t* indices, uint32_t* n_cells_out, int* dense_out) {
  MgSim* s = nullptr;
  uint32_t res[9] = {};
  int rc = probe(xy, n, cell, 0, &s, res);
  if (rc) return rc;
  *dense_out = (int)res[0];
  min_cxy[0] = (int32_t)res[1];
  min_cxy[1] = (int32_t)res[2];
  wh[0] = res[0] ? (int64_t)(int32_t)res[3] : 0;
  wh[1] = res[0] ? (int64_t)(int32_t)res[4] : 0;
  uint32_t nc = res[6] ? res[5] : 0;
  *n_cells_out = nc + 1;
  if (nc + 1 > cell_cap) { mg_sim_destroy(s); return fail_global(MG_ERR_CAPACITY, "cell buffer too small"); }
  cudaMemcpy(cell_start, s->md.gA.cell_start, 4 * ((size_t)nc + 1), cudaMemcpyDeviceToHost);
  if (n) cudaMemcpy(indices, s->md.gA.indices, 4 * (size_t)res[6], cudaMemcpyDeviceToHost);
  mg_sim_destroy(s);
  return MG_OK;
}
int mg_probe_candidate_pairs(const float* xy, uint32_t n, float cell, uint32_t* pairs, uint32_t cap, uint32_t* n_out) {
  MgSim* s = nullptr;
  uint32_t res[9] = {};
  int rc = probe(xy, n, cell, 1, &s, res);
  if (rc) return rc;
  uint32_t np = res[8];
  *n_out = np;
  if (res[7]) { mg_sim_destroy(s); return fail_global(MG_ERR_CAPACITY, "probe error bits 0x%x", res[7]); }
  if (np > cap) { mg_sim_destroy(s); return fail_global(MG_ERR_CAPACITY, "pair buffer too small"); }
  std::vector<uint32_t> pi(np), pj(np);
  if (np) {
    cudaMemcpy(pi.data(), s->md.pair_i, 4 * (size_t)np, cudaMemcpyDeviceToHost);
    cudaMemcpy(pj.data(), s->md.pair_j, 4 * (size_t)np, cudaMemcpyDeviceToHost);
  }
  for (uint32_t k = 0; k < np; ++k) { pairs[2 * k] = pi[k]; pairs[2 * k + 1] = pj[k]; }
  mg_sim_destroy(s);
  return MG_OK;
}
int mg_probe_neighbor_lists(const float* xy, uint32_t n, float h, uint32_t* offsets, uint32_t* nbrs, uint32_t cap,
                            uint32_t* n_edges) {
  MgSim* s = nullptr;
  uint32_t res[9] = {};
  int rc = probe(xy, n, h, 2, &s, res);
  if (rc) return rc;
  uint32_t ne = res[8];
  *n_edges = ne;
  if (res[7]) { mg_sim_destroy(s); return fail_global(MG_ERR_CAPACITY, "probe error bits 0x%x", res[7]); }
  cudaMemcpy(offsets, s->md.nbr_off, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost);
  if (ne > cap) { mg_sim_destroy(s); return fail_global(MG_ERR_CAPACITY, "neighbour buffer too small"); }
  if (ne) cudaMemcpy(nbrs, s->md.nbrs, 4 * (size_t)ne, cudaMemcpyDeviceToHost);
  mg_sim_destroy(s);
  return MG_OK;
}

}  // extern "C"

// ====================================================================== batches of mills
// Many independent mills advanced together: one launch per frame with one thread block per mill
// (each mill its own sub-step count), then one packing launch for the impact records. Every mill
// keeps the arena, uniforms and host bookkeeping of an ordinary handle (EMA power and torque,
// energy budget, stress accumulators), so a mill's results are the same alone or in a batch.
struct MgBatch {
  std::vector<MgSim*> mills;
  std::vector<uint32_t> n_sub;  // effective_substeps per mill
  uint32_t stride = 0;          // sub-step stride of the angle and output blocks (max n_sub)
  cudaStream_t stream = nullptr;
  MillDev* d_md = nullptr;      // descriptors (out -> the batch's output block)
  StepUniform* d_uni = nullptr;
  SubAngles* d_ang = nullptr;
  SubAngles* h_ang = nullptr;
  uint32_t* d_nsub = nullptr;
  StepOut* d_out = nullptr;
  StepOut* h_out = nullptr;
  MgImpactRecord* d_packed = nullptr;
  MgImpactRecord* h_packed = nullptr;
  uint32_t packed_cap = 0;
  uint32_t* d_cursor = nullptr;
  uint2* d_table = nullptr;
  uint2* h_table = nullptr;
  size_t smem = 0;
  uint32_t threads = 0;
  bool regs64 = false;
  // blocks run the mills longest first (block k -> mill order[k]): the cost of a mill is its
  // device cycles in the last frame (an estimate from its sizes before the first one)
  std::vector<uint32_t> order;
  std::vector<double> cost;
  uint32_t* d_order = nullptr;
  // the mills' stress-accumulator states after each launch (one block, copied back at once)
  StressState* d_stress = nullptr;
  StressState* h_stress = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_kernel_ms = 0.0f;
  uint64_t launches = 0;
  std::string err;
};

namespace {

int bfail(MgBatch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  g_err = buf;
  return code;
}
#define BCK(call)                                                                   \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return bfail(b, MG_ERR_CUDA, "%s", cudaGetErrorString(e_)); \
  } while (0)

// Uploads the descriptors and mill-uniform blocks of every mill (at creation and after options
// change).
// Runs f(i) for i in [0, n) on up to 16 host threads (each i once; the calls must be
// independent).
template <class F>
void parallel_for(uint32_t n, F f) {
  const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t t = std::min<uint32_t>({16u, hw, (n + 31u) / 32u});
  if (t <= 1) {
    for (uint32_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> pool;
  for (uint32_t w = 0; w < t; ++w)
    pool.emplace_back([&, w]() {
      for (uint32_t i = w; i < n; i += t) f(i);
    });
  for (std::thread& th : pool) th.join();
}

// The mills' block order, longest first; uploaded when it changed.
int batch_order(MgBatch* b) {
  const uint32_t n = (uint32_t)b->mills.size();
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return b->cost[x] > b->cost[y]; });
  if (order == b->order) return MG_OK;
  b->order = order;
  BCK(cudaMemcpyAsync(b->d_order, b->order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, b->stream));
  return MG_OK;
}

int batch_upload(MgBatch* b) {
  const uint32_t n = (uint32_t)b->mills.size();
  std::vector<MillDev> md(n);
  std::vector<StepUniform> uni(n);
  b->smem = 0;
  for (uint32_t i = 0; i < n; ++i) {
    MgSim* s = b->mills[i];
    const MgSimulationParams& q = s->params.simulation;
    int rc = fill_uniform(s, sim_drum(s), s->params.media, s->params.slurry, q.pbf_iterations, q.dem_iterations, 1,
                          1, 1);
    if (rc) return bfail(b, rc, "mill %u: %s", i, s->err.c_str());
    fill_desc(s);
    md[i] = s->md;
    md[i].out = b->d_out + (size_t)i * b->stride;
    md[i].stress_copy = b->d_stress + i;
    uni[i] = *s->h_uni;
    uni[i].fold_stress = 1u;
    b->smem = std::max(b->smem, (size_t)s->md.smem_bytes);
  }
  BCK(cudaMemcpyAsync(b->d_md, md.data(), sizeof(MillDev) * n, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->d_uni, uni.data(), sizeof(StepUniform) * n, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return MG_OK;
}

}  // namespace

extern "C" {

int mg_batch_create(const MgParams* params, uint32_t n_mills, MgBatch** out) {
  if (!params || !out || n_mills == 0) return fail_global(MG_ERR_ARG, "null argument or empty batch");
  MgBatch* b = new MgBatch();
  int rc = MG_OK;
  for (uint32_t i = 0; i < n_mills && !rc; ++i) {
    MgSim* s = nullptr;
    rc = create_sim(&params[i], nullptr, 0, &s);
    if (rc) { bfail(b, rc, "mill %u: %s", i, g_err.c_str()); break; }
    b->mills.push_back(s);
    uint32_t ns = std::max(mgh::effective_substeps(s->params), 1u);
    if (ns > MAX_SUB) { rc = bfail(b, MG_ERR_ARG, "mill %u: %u sub-steps per frame, at most %u", i, ns, MAX_SUB); break; }
    b->n_sub.push_back(ns);
    b->stride = std::max(b->stride, ns);
  }
  auto setup = [&]() -> int {
    BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCK(cudaMalloc(&b->d_md, sizeof(MillDev) * n_mills));
    BCK(cudaMalloc(&b->d_uni, sizeof(StepUniform) * n_mills));
    BCK(cudaMalloc(&b->d_ang, sizeof(SubAngles) * n_mills * b->stride));
    BCK(cudaMallocHost(&b->h_ang, sizeof(SubAngles) * n_mills * b->stride));
    BCK(cudaMalloc(&b->d_nsub, sizeof(uint32_t) * n_mills));
    BCK(cudaMalloc(&b->d_out, sizeof(StepOut) * n_mills * b->stride));
    BCK(cudaMallocHost(&b->h_out, sizeof(StepOut) * n_mills * b->stride));
    uint64_t cap = 0;
    for (MgSim* s : b->mills) cap += (uint64_t)s->md.cap_impacts * b->stride;
    b->packed_cap = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFF0ull);
    BCK(cudaMalloc(&b->d_packed, sizeof(MgImpactRecord) * (size_t)b->packed_cap));
    BCK(cudaMallocHost(&b->h_packed, sizeof(MgImpactRecord) * (size_t)b->packed_cap));
    BCK(cudaMalloc(&b->d_cursor, sizeof(uint32_t)));
    BCK(cudaMalloc(&b->d_table, sizeof(uint2) * n_mills));
    BCK(cudaMallocHost(&b->h_table, sizeof(uint2) * n_mills));
    BCK(cudaEventCreate(&b->ev0));
    BCK(cudaEventCreate(&b->ev1));
    BCK(cudaMalloc(&b->d_order, sizeof(uint32_t) * n_mills));
    BCK(cudaMalloc(&b->d_stress, sizeof(StressState) * n_mills));
    BCK(cudaMallocHost(&b->h_stress, sizeof(StressState) * n_mills));
    BCK(cudaMemcpyAsync(b->d_nsub, b->n_sub.data(), sizeof(uint32_t) * n_mills, cudaMemcpyHostToDevice, b->stream));
    // before the first frame: sub-steps times particles, balls weighted for their sweeps
    b->cost.resize(n_mills);
    for (uint32_t i = 0; i < n_mills; ++i)
      b->cost[i] = (double)b->n_sub[i] * ((double)b->mills[i]->nf + 4.0 * (double)b->mills[i]->nb);
    int orc = batch_order(b);
    if (orc) return orc;
    return batch_upload(b);
  };
  if (!rc) rc = setup();
  if (rc) {
    std::string e = b->err;
    mg_batch_destroy(b);
    g_err = e;
    return rc;
  }
  *out = b;
  return MG_OK;
}

void mg_batch_destroy(MgBatch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (MgSim* s : b->mills) mg_sim_destroy(s);
  if (b->d_md) cudaFree(b->d_md);
  if (b->d_uni) cudaFree(b->d_uni);
  if (b->d_ang) cudaFree(b->d_ang);
  if (b->h_ang) cudaFreeHost(b->h_ang);
  if (b->d_nsub) cudaFree(b->d_nsub);
  if (b->d_out) cudaFree(b->d_out);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->d_packed) cudaFree(b->d_packed);
  if (b->h_packed) cudaFreeHost(b->h_packed);
  if (b->d_cursor) cudaFree(b->d_cursor);
  if (b->d_table) cudaFree(b->d_table);
  if (b->h_table) cudaFreeHost(b->h_table);
  if (b->d_order) cudaFree(b->d_order);
  if (b->d_stress) cudaFree(b->d_stress);
  if (b->h_stress) cudaFreeHost(b->h_stress);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char* mg_batch_last_error(const MgBatch* b) { return b ? b->err.c_str() : g_err.c_str(); }

uint32_t mg_batch_size(const MgBatch* b) { return b ? (uint32_t)b->mills.size() : 0u; }

int mg_batch_set_options(MgBatch* b, const MgOptions* opt) {
  if (!b || !opt) return fail_global(MG_ERR_ARG, "null argument");
  for (MgSim* s : b->mills) {
    int rc = mg_sim_set_options(s, opt);
    if (rc) return bfail(b, rc, "%s", s->err.c_str());
  }
  b->threads = opt->block_threads;
  b->regs64 = opt->block_regs == 64;
  return batch_upload(b);
}

int mg_batch_mill(MgBatch* b, uint32_t i, MgSim** out) {
  if (!b || !out) return fail_global(MG_ERR_ARG, "null argument");
  if (i >= b->mills.size()) return bfail(b, MG_ERR_ARG, "mill %u out of range (%zu mills)", i, b->mills.size());
  *out = b->mills[i];
  return MG_OK;
}

int mg_batch_step_frames(MgBatch* b, uint32_t frames, float frame_dt) {
  if (!b) return fail_global(MG_ERR_ARG, "null handle");
  const uint32_t n = (uint32_t)b->mills.size();
  // descriptors follow the members' current counts and materials (the per-mill setters may change
  // them between calls)
  std::vector<MillDev> md(n);
  for (uint32_t i = 0; i < n; ++i) {
    MgSim* s = b->mills[i];
    int rc = check_materials(s);
    if (rc) return bfail(b, rc, "mill %u: %s", i, s->err.c_str());
    fill_desc(s);
    md[i] = s->md;
    md[i].out = b->d_out + (size_t)i * b->stride;
    md[i].stress_copy = b->d_stress + i;
    b->smem = std::max(b->smem, (size_t)s->md.smem_bytes);
  }
  BCK(cudaMemcpyAsync(b->d_md, md.data(), sizeof(MillDev) * n, cudaMemcpyHostToDevice, b->stream));
  for (uint32_t f = 0; f < frames; ++f) {
    // Simulation::step(frame_dt) for every mill: n_sub[i] sub-steps of frame_dt / n_sub[i]
    for (uint32_t i = 0; i < n; ++i) {
      MgSim* s = b->mills[i];
      const uint32_t ns = b->n_sub[i];
      const float sub_dt = frame_dt / (float)ns;
      const float omega = mgh::mill_omega(s->params.mill);
      float angle = s->drum_angle;
      double now = s->sim_time;
      for (uint32_t k = 0; k < ns; ++k) {
        fill_angle(b->h_ang[(size_t)i * b->stride + k], angle, omega, sub_dt, now);
        angle = mgh::rem_euclid_r(angle + omega * sub_dt, mgh::TAU_F);
        now += (double)sub_dt;
      }
    }
    BCK(cudaMemcpyAsync(b->d_ang, b->h_ang, sizeof(SubAngles) * n * b->stride, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaEventRecord(b->ev0, b->stream));
    int orc = batch_order(b);
    if (orc) return orc;
    BCK(launch_substeps(b->d_md, n, b->d_uni, b->d_ang, b->stride, b->d_nsub, b->threads, b->smem, b->stream, 1,
                        b->d_order, b->regs64));
    BCK(cudaEventRecord(b->ev1, b->stream));
    BCK(cudaMemsetAsync(b->d_cursor, 0, sizeof(uint32_t), b->stream));
    BCK(launch_pack_impacts(b->d_md, n, b->d_nsub, b->d_packed, b->packed_cap, b->d_cursor, b->d_table, b->stream));
    BCK(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(StepOut) * n * b->stride, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaMemcpyAsync(b->h_table, b->d_table, sizeof(uint2) * n, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaMemcpyAsync(b->h_stress, b->d_stress, sizeof(StressState) * n, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    BCK(cudaEventElapsedTime(&b->last_kernel_ms, b->ev0, b->ev1));
    b->launches += 1;
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) total = std::max<uint64_t>(total, (uint64_t)b->h_table[i].x + b->h_table[i].y);
    if (total > b->packed_cap) return bfail(b, MG_ERR_CAPACITY, "impact records exceed the batch buffer");
    if (total)
      BCK(cudaMemcpyAsync(b->h_packed, b->d_packed, sizeof(MgImpactRecord) * total, cudaMemcpyDeviceToHost,
                          b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (uint32_t i = 0; i < n; ++i) {
      const StepOut* o = b->h_out + (size_t)i * b->stride;
      uint32_t e = 0;
      for (uint32_t k = 0; k < b->n_sub[i]; ++k) e |= o[k].err;
      if (e) return bfail(b, MG_ERR_CAPACITY, "mill %u: device capacity exceeded (error bits 0x%x)", i, e);
    }
    // the mills' host folds (EMA, energy budget, stress accumulator) are independent of one
    // another: they run on several host threads
    parallel_for(n, [&](uint32_t i) {
      MgSim* s = b->mills[i];
      const uint32_t ns = b->n_sub[i];
      const StepOut* o = b->h_out + (size_t)i * b->stride;
      double cyc = 0.0;
      for (uint32_t k = 0; k < ns; ++k)
        for (int q = 0; q <= 14; ++q) cyc += (double)o[k].stage[q];
      b->cost[i] = cyc;
      s->stress = b->h_stress[i];
      std::memcpy(s->h_out, o, sizeof(StepOut) * ns);
      const MgImpactRecord* rec = b->h_packed + b->h_table[i].x;
      for (uint32_t k = 0; k < ns; ++k) {
        const uint32_t ni = std::min(o[k].n_impacts, s->md.cap_impacts);
        if (ni) std::memcpy(s->h_imp + (size_t)k * s->md.cap_impacts, rec, sizeof(MgImpactRecord) * ni);
        rec += ni;
        const uint32_t* c = reinterpret_cast<const uint32_t*>(&o[k].ctr);
        for (int q = 0; q < 10; ++q) s->ctr_tot[q] += c[q];
        for (int q = 0; q < 40; ++q) s->stage_tot[q] += o[k].stage[q];
        s->ctr_n += 1;
      }
      s->max_disp = 0.0f;
      s->clamp_hits_frame = 0;
      const float sub_dt = frame_dt / (float)ns;
      const float omega = mgh::mill_omega(s->params.mill);
      for (uint32_t k = 0; k < ns; ++k) fold_substep(s, k, sub_dt, omega);
      s->last_fluid = o[ns - 1].fs;
      s->last_dem = o[ns - 1].ds;
      s->last_ctr = o[ns - 1].ctr;
      s->launches += 1;
    });
  }
  return MG_OK;
}

int mg_batch_scalars(MgBatch* b, MgScalars* out) {
  if (!b || !out) return fail_global(MG_ERR_ARG, "null argument");
  for (size_t i = 0; i < b->mills.size(); ++i) {
    int rc = mg_get_scalars(b->mills[i], &out[i]);
    if (rc) return bfail(b, rc, "mill %zu: %s", i, b->mills[i]->err.c_str());
  }
  return MG_OK;
}

int mg_batch_stream(MgBatch* b, void** stream) {
  if (!b || !stream) return fail_global(MG_ERR_ARG, "null argument");
  *stream = b->stream;
  return MG_OK;
}

int mg_batch_last_kernel_ms(MgBatch* b, float* ms, uint64_t* launches) {
  if (!b) return fail_global(MG_ERR_ARG, "null handle");
  if (ms) *ms = b->last_kernel_ms;
  if (launches) *launches = b->launches;
  return MG_OK;
}

int mg_sim_footprint(const MgSim* s, uint64_t* device_bytes) {
  if (!s || !device_bytes) return fail_global(MG_ERR_ARG, "null argument");
  *device_bytes = (uint64_t)s->dbytes + sizeof(MillDev) + sizeof(StepUniform) + sizeof(SubAngles) * MAX_SUB;
  return MG_OK;
}

}  // extern "C"

// ====================================================================== request server
// Continuous batching of mill jobs: submitted jobs wait in a queue and are admitted, oldest first,
// whenever the device bytes their arenas need fit under the budget; every step advances all
// admitted jobs by one frame in one launch (one thread block per job, each its own sub-step
// count) and retires the jobs that reached their horizon, freeing their memory for the queue.
// A job advances exactly as the same mill stepped alone (the same kernels on the same state), so
// its results do not depend on what else is in the mix.
struct SeedAcc;  // run_seed's window accumulators (with the grinding statistics below)
bool seed_window(const MgParams& p, float warmup_revolutions, float measure_revolutions, uint32_t* warm,
                 uint32_t* meas, double* rev_s);
SeedAcc* seed_acc_new(const MgParams& p, uint32_t warm, uint32_t meas, double rev_s);
void seed_acc_free(SeedAcc* a);
void seed_acc_observe(SeedAcc* a, const MgSim* s, uint32_t frames_done);
void seed_acc_finish(const SeedAcc* a, const MgSim* s, MgSeedResult* r);

struct MgServerJob {
  uint64_t id = 0;
  MgParams params{};
  uint32_t frames_total = 0, frames_done = 0, n_sub = 0;
  MgSim* sim = nullptr;
  uint64_t bytes = 0;
  bool cancel = false;
  double t_submit = 0.0, t_admit = 0.0, t_first = -1.0;
  // a seed of a sweep: the sweep's id, the seed's index in it and its run_seed window
  uint64_t sweep = 0;
  uint32_t sweep_index = 0;
  SeedAcc* acc = nullptr;
  double cost = -1.0;  // device cycles of the job's last frame (its block order in the launch)
};

// A seed-sweep job: one server job per seed, combined when all have finished.
struct MgServerSweep {
  uint32_t n_seeds = 0, finished = 0, state = MG_JOB_QUEUED;
  std::vector<MgSeedResult> results;
};

struct MgServer {
  MgServerConfig cfg{};
  std::string err;
  cudaStream_t stream = nullptr;
  std::deque<MgServerJob*> queue;
  std::vector<MgServerJob*> active;
  std::vector<MgJobUpdate> pending;
  std::map<uint64_t, MgServerSweep> sweeps;
  uint64_t next_id = 1, in_use = 0, frames = 0;
  uint32_t finished_total = 0;
  // launch blocks, grown as needed (cap jobs, MAX_SUB sub-steps each)
  uint32_t cap = 0;
  MillDev *d_md = nullptr, *h_md = nullptr;
  StepUniform *d_uni = nullptr, *h_uni = nullptr;
  SubAngles *d_ang = nullptr, *h_ang = nullptr;
  uint32_t *d_nsub = nullptr, *h_nsub = nullptr;
  StepOut *d_out = nullptr, *h_out = nullptr;
  uint2 *d_table = nullptr, *h_table = nullptr;
  uint32_t *d_order = nullptr, *h_order = nullptr;  // block k runs job h_order[k] (longest first)
  StressState *d_stress = nullptr, *h_stress = nullptr;  // the jobs' stress states after a launch
  uint32_t* d_cursor = nullptr;
  MgImpactRecord *d_packed = nullptr, *h_packed = nullptr;
  uint64_t packed_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_kernel_ms = 0.0f, last_frame_ms = 0.0f;
};

namespace {

double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int sfail(MgServer* v, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (v) v->err = buf;
  g_err = buf;
  return code;
}
#define SCK(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return sfail(v, MG_ERR_CUDA, "%s", cudaGetErrorString(e_));   \
  } while (0)

void server_free_blocks(MgServer* v) {
  cudaFree(v->d_md); cudaFreeHost(v->h_md);
  cudaFree(v->d_uni); cudaFreeHost(v->h_uni);
  cudaFree(v->d_ang); cudaFreeHost(v->h_ang);
  cudaFree(v->d_nsub); cudaFreeHost(v->h_nsub);
  cudaFree(v->d_out); cudaFreeHost(v->h_out);
  cudaFree(v->d_table); cudaFreeHost(v->h_table);
  cudaFree(v->d_order); cudaFreeHost(v->h_order);
  v->d_order = v->h_order = nullptr;
  cudaFree(v->d_stress); cudaFreeHost(v->h_stress);
  v->d_stress = v->h_stress = nullptr;
  v->d_md = v->h_md = nullptr;
  v->d_uni = v->h_uni = nullptr;
  v->d_ang = v->h_ang = nullptr;
  v->d_nsub = v->h_nsub = nullptr;
  v->d_out = v->h_out = nullptr;
  v->d_table = v->h_table = nullptr;
  v->cap = 0;
}

int server_reserve(MgServer* v, uint32_t n, uint64_t packed) {
  if (n > v->cap) {
    SCK(cudaStreamSynchronize(v->stream));
    server_free_blocks(v);
    const uint32_t c = std::max(n, 2 * v->cap);
    SCK(cudaMalloc(&v->d_md, sizeof(MillDev) * c));
    SCK(cudaMallocHost(&v->h_md, sizeof(MillDev) * c));
    SCK(cudaMalloc(&v->d_uni, sizeof(StepUniform) * c));
    SCK(cudaMallocHost(&v->h_uni, sizeof(StepUniform) * c));
    SCK(cudaMalloc(&v->d_ang, sizeof(SubAngles) * c * MAX_SUB));
    SCK(cudaMallocHost(&v->h_ang, sizeof(SubAngles) * c * MAX_SUB));
    SCK(cudaMalloc(&v->d_nsub, sizeof(uint32_t) * c));
    SCK(cudaMallocHost(&v->h_nsub, sizeof(uint32_t) * c));
    SCK(cudaMalloc(&v->d_out, sizeof(StepOut) * c * MAX_SUB));
    SCK(cudaMallocHost(&v->h_out, sizeof(StepOut) * c * MAX_SUB));
    SCK(cudaMalloc(&v->d_table, sizeof(uint2) * c));
    SCK(cudaMallocHost(&v->h_table, sizeof(uint2) * c));
    SCK(cudaMalloc(&v->d_order, sizeof(uint32_t) * c));
    SCK(cudaMallocHost(&v->h_order, sizeof(uint32_t) * c));
    SCK(cudaMalloc(&v->d_stress, sizeof(StressState) * c));
    SCK(cudaMallocHost(&v->h_stress, sizeof(StressState) * c));
    v->cap = c;
  }
  if (packed > v->packed_cap) {
    SCK(cudaStreamSynchronize(v->stream));
    cudaFree(v->d_packed);
    cudaFreeHost(v->h_packed);
    v->d_packed = v->h_packed = nullptr;
    const uint64_t c = std::max<uint64_t>(packed, 2 * v->packed_cap);
    SCK(cudaMalloc(&v->d_packed, sizeof(MgImpactRecord) * c));
    SCK(cudaMallocHost(&v->h_packed, sizeof(MgImpactRecord) * c));
    v->packed_cap = c;
  }
  return MG_OK;
}

MgJobUpdate job_update(const MgServerJob* j, uint32_t state) {
  MgJobUpdate u;
  std::memset(&u, 0, sizeof(u));
  u.job_id = j->id;
  u.state = state;
  u.frames_done = j->frames_done;
  u.frames_total = j->frames_total;
  u.queued_s = j->t_admit > 0.0 ? j->t_admit - j->t_submit : 0.0;
  u.first_frame_s = j->t_first >= 0.0 ? j->t_first - j->t_submit : 0.0;
  if (j->sim) {
    mg_get_scalars(j->sim, &u.scalars);
    mg_stress_histogram_rate(j->sim, u.stress_histogram_rate);
  }
  return u;
}

void retire(MgServer* v, MgServerJob* j, uint32_t state) {
  MgJobUpdate u = job_update(j, state);
  if (j->sim && state == MG_JOB_FINISHED) mg_state_hash(j->sim, 1, &u.state_hash);
  v->pending.push_back(u);
  auto sit = j->sweep ? v->sweeps.find(j->sweep) : v->sweeps.end();
  if (sit != v->sweeps.end()) {
    MgServerSweep& sw = sit->second;
    if (state == MG_JOB_FINISHED && j->sim && j->acc) {
      seed_acc_finish(j->acc, j->sim, &sw.results[j->sweep_index]);
      sw.finished += 1;
      if (sw.finished == sw.n_seeds && sw.state != MG_JOB_CANCELLED && sw.state != MG_JOB_FAILED)
        sw.state = MG_JOB_FINISHED;
    } else if (sw.state != MG_JOB_FAILED) {
      sw.state = state == MG_JOB_FAILED ? MG_JOB_FAILED : MG_JOB_CANCELLED;
    }
    if (state != MG_JOB_FINISHED) {
      // the sweep cannot finish any more: its other seeds leave too (queued ones at the next
      // admission, running ones before the next frame) instead of holding slots and memory
      for (MgServerJob* o : v->queue)
        if (o->sweep == j->sweep) o->cancel = true;
      for (MgServerJob* o : v->active)
        if (o->sweep == j->sweep) o->cancel = true;
    }
  }
  if (j->acc) {
    seed_acc_free(j->acc);
    j->acc = nullptr;
  }
  if (j->sim) {
    mg_sim_destroy(j->sim);
    v->in_use -= j->bytes;
  }
  v->finished_total += 1;
  delete j;
}

}  // namespace

extern "C" {

int mg_server_create(const MgServerConfig* cfg, MgServer** out) {
  if (!out) return fail_global(MG_ERR_ARG, "null argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail_global(MG_ERR_NO_DEVICE, "no CUDA device visible");
  MgServer* v = new MgServer();
  if (cfg) v->cfg = *cfg;
  if (v->cfg.memory_budget_bytes == 0) v->cfg.memory_budget_bytes = 150ull << 30;
  if (v->cfg.max_active == 0) v->cfg.max_active = 1024;
  if (!(v->cfg.frame_dt > 0.0f)) v->cfg.frame_dt = 1.0f / 60.0f;
  if (v->cfg.block_threads != 0 && (v->cfg.block_threads % 32 != 0 || v->cfg.block_threads > MAX_BLOCK_THREADS)) {
    delete v;
    return fail_global(MG_ERR_ARG, "block_threads must be a multiple of 32 in [32, %u]", MAX_BLOCK_THREADS);
  }
  auto setup = [&]() -> int {
    SCK(cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking));
    SCK(cudaEventCreate(&v->ev0));
    SCK(cudaEventCreate(&v->ev1));
    SCK(cudaMalloc(&v->d_cursor, sizeof(uint32_t)));
    // retired jobs' arenas stay in the device pool for the next admissions
    int dev = 0;
    SCK(cudaGetDevice(&dev));
    cudaMemPool_t pool;
    SCK(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t keep = v->cfg.memory_budget_bytes;
    SCK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    return MG_OK;
  };
  int rc = setup();
  if (rc) {
    std::string e = v->err;
    mg_server_destroy(v);
    g_err = e;
    return rc;
  }
  *out = v;
  return MG_OK;
}

void mg_server_destroy(MgServer* v) {
  if (!v) return;
  if (v->stream) cudaStreamSynchronize(v->stream);
  for (MgServerJob* j : v->active) {
    if (j->sim) mg_sim_destroy(j->sim);
    delete j;
  }
  for (MgServerJob* j : v->queue) delete j;
  if (v->stream) cudaStreamSynchronize(v->stream);
  server_free_blocks(v);
  cudaFree(v->d_packed);
  cudaFreeHost(v->h_packed);
  cudaFree(v->d_cursor);
  if (v->ev0) cudaEventDestroy(v->ev0);
  if (v->ev1) cudaEventDestroy(v->ev1);
  if (v->stream) cudaStreamDestroy(v->stream);
  delete v;
}

const char* mg_server_last_error(const MgServer* v) { return v ? v->err.c_str() : g_err.c_str(); }

int mg_server_submit(MgServer* v, const MgParams* p, double horizon_s, uint64_t* job_id) {
  if (!v || !p) return fail_global(MG_ERR_ARG, "null argument");
  std::string e;
  if (!mgh::params_validate(*p, &e)) return sfail(v, MG_ERR_INVALID_PARAMS, "%s", e.c_str());
  if (!(horizon_s > 0.0) || !std::isfinite(horizon_s)) return sfail(v, MG_ERR_ARG, "horizon must be positive");
  const uint32_t ns = std::max(mgh::effective_substeps(*p), 1u);
  if (ns > MAX_SUB) return sfail(v, MG_ERR_ARG, "%u sub-steps per frame, at most %u", ns, MAX_SUB);
  MgServerJob* j = new MgServerJob();
  j->id = v->next_id++;
  j->params = *p;
  j->n_sub = ns;
  j->frames_total = (uint32_t)std::max(1.0, std::ceil(horizon_s / (double)v->cfg.frame_dt - 1e-9));
  j->t_submit = wall_s();
  v->queue.push_back(j);
  if (job_id) *job_id = j->id;
  return MG_OK;
}

// The web batch planner's repeat runs (web/src/batch/plan.ts:5-33, 78-91; protocol.ts): seeds
// 1..=n_seeds of the same Params, each batch::run_seed over the same window, then combine.
int mg_server_submit_sweep(MgServer* v, const MgParams* p, uint32_t n_seeds, float warmup_revolutions,
                           float measure_revolutions, uint64_t* sweep_id) {
  if (!v || !p) return fail_global(MG_ERR_ARG, "null argument");
  std::string e;
  if (!mgh::params_validate(*p, &e)) return sfail(v, MG_ERR_INVALID_PARAMS, "%s", e.c_str());
  if (n_seeds < 1 || n_seeds > MG_SWEEP_MAX_SEEDS)
    return sfail(v, MG_ERR_ARG, "seeds must be from 1 to %u", (unsigned)MG_SWEEP_MAX_SEEDS);
  if (!(measure_revolutions >= 1.0f) || measure_revolutions != std::floor(measure_revolutions))
    return sfail(v, MG_ERR_ARG, "measured revolutions must be an integer >= 1");
  if (!(warmup_revolutions >= 0.0f) || !std::isfinite(warmup_revolutions))
    return sfail(v, MG_ERR_ARG, "warm-up revolutions must be a number >= 0");
  if (!(mgh::mill_rpm(p->mill) > 0.0f))
    return sfail(v, MG_ERR_ARG, "the drum speed is 0; whole-revolution windows are undefined");
  const float k = mgh::effective_media(*p).scale_factor;
  if (k > 1.0f)
    return sfail(v, MG_ERR_ARG,
                 "coarse-graining is active (k = %.2f): the statistics are meaningless; raise max balls so that k = 1",
                 k);
  const uint32_t ns = std::max(mgh::effective_substeps(*p), 1u);
  if (ns > MAX_SUB) return sfail(v, MG_ERR_ARG, "%u sub-steps per frame, at most %u", ns, MAX_SUB);
  uint32_t warm = 0, meas = 0;
  double rev_s = 0.0;
  if (!seed_window(*p, warmup_revolutions, measure_revolutions, &warm, &meas, &rev_s))
    return sfail(v, MG_ERR_ARG, "invalid revolutions");
  const uint64_t id = v->next_id++;
  MgServerSweep& sw = v->sweeps[id];
  sw.n_seeds = n_seeds;
  sw.results.assign(n_seeds, MgSeedResult{});
  for (uint32_t i = 0; i < n_seeds; ++i) {
    MgServerJob* j = new MgServerJob();
    j->id = v->next_id++;
    j->params = *p;
    j->params.simulation.seed = i + 1;  // the literal numbers 1..N (plan.ts:29-32)
    j->n_sub = ns;
    j->frames_total = warm + meas;
    j->t_submit = wall_s();
    j->sweep = id;
    j->sweep_index = i;
    j->acc = seed_acc_new(j->params, warm, meas, rev_s);
    v->queue.push_back(j);
  }
  if (sweep_id) *sweep_id = id;
  return MG_OK;
}

int mg_server_sweep_result(MgServer* v, uint64_t sweep_id, MgSeedResult* results, double* mean, double* std_err,
                           uint32_t* state, uint32_t* seeds_finished) {
  if (!v) return fail_global(MG_ERR_ARG, "null handle");
  auto it = v->sweeps.find(sweep_id);
  if (it == v->sweeps.end()) return sfail(v, MG_ERR_ARG, "no sweep %llu", (unsigned long long)sweep_id);
  const MgServerSweep& sw = it->second;
  if (state) *state = sw.state;
  if (seeds_finished) *seeds_finished = sw.finished;
  if (sw.state != MG_JOB_FINISHED) return MG_OK;
  if (results) std::memcpy(results, sw.results.data(), sizeof(MgSeedResult) * sw.n_seeds);
  if (mean && std_err) return mg_seed_combine(sw.results.data(), sw.n_seeds, mean, std_err);
  return MG_OK;
}

int mg_server_sweep_release(MgServer* v, uint64_t sweep_id) {
  if (!v) return fail_global(MG_ERR_ARG, "null handle");
  auto it = v->sweeps.find(sweep_id);
  if (it == v->sweeps.end()) return sfail(v, MG_ERR_ARG, "no sweep %llu", (unsigned long long)sweep_id);
  for (MgServerJob* j : v->queue)
    if (j->sweep == sweep_id) j->cancel = true;
  for (MgServerJob* j : v->active)
    if (j->sweep == sweep_id) j->cancel = true;
  v->sweeps.erase(it);
  return MG_OK;
}

int mg_server_cancel(MgServer* v, uint64_t job_id) {
  if (!v) return fail_global(MG_ERR_ARG, "null handle");
  auto sw = v->sweeps.find(job_id);
  if (sw != v->sweeps.end()) {
    // every seed of the sweep still queued or running
    std::vector<uint64_t> ids;
    for (MgServerJob* j : v->queue)
      if (j->sweep == job_id) ids.push_back(j->id);
    for (MgServerJob* j : v->active)
      if (j->sweep == job_id) ids.push_back(j->id);
    for (uint64_t id : ids) mg_server_cancel(v, id);
    if (sw->second.state != MG_JOB_FINISHED) sw->second.state = MG_JOB_CANCELLED;
    return MG_OK;
  }
  for (auto it = v->queue.begin(); it != v->queue.end(); ++it) {
    if ((*it)->id == job_id) {
      MgServerJob* j = *it;
      v->queue.erase(it);
      retire(v, j, MG_JOB_CANCELLED);
      return MG_OK;
    }
  }
  for (MgServerJob* j : v->active)
    if (j->id == job_id) { j->cancel = true; return MG_OK; }
  return sfail(v, MG_ERR_ARG, "no queued or running job %llu", (unsigned long long)job_id);
}

int mg_server_step(MgServer* v) {
  if (!v) return fail_global(MG_ERR_ARG, "null handle");
  const double t0 = wall_s();
  // cancelled jobs leave before the frame
  for (size_t k = 0; k < v->active.size();) {
    if (v->active[k]->cancel) {
      retire(v, v->active[k], MG_JOB_CANCELLED);
      v->active.erase(v->active.begin() + (long)k);
    } else {
      ++k;
    }
  }
  // admission, oldest first, by the device bytes each job's arena needs
  while (!v->queue.empty() && v->active.size() < v->cfg.max_active) {
    MgServerJob* j = v->queue.front();
    if (j->cancel) {  // a seed of a sweep that failed or was released
      v->queue.pop_front();
      retire(v, j, MG_JOB_CANCELLED);
      continue;
    }
    MgSim* sim = nullptr;
    int rc = create_sim(&j->params, nullptr, 0, &sim, v->stream);
    if (!rc) rc = check_materials(sim);
    if (rc) {
      if (sim) mg_sim_destroy(sim);
      v->queue.pop_front();
      retire(v, j, MG_JOB_FAILED);
      continue;
    }
    const uint64_t need = sim->dbytes;
    if (v->in_use + need > v->cfg.memory_budget_bytes) {
      mg_sim_destroy(sim);
      if (v->active.empty()) {  // it could never fit
        v->queue.pop_front();
        retire(v, j, MG_JOB_FAILED);
        continue;
      }
      break;  // wait for running jobs to free memory
    }
    j->sim = sim;
    j->bytes = need;
    j->t_admit = wall_s();
    if (j->acc) {
      seed_acc_observe(j->acc, sim, 0);  // the window's start when there is no warm-up
      auto sit = v->sweeps.find(j->sweep);
      if (sit != v->sweeps.end() && sit->second.state == MG_JOB_QUEUED) sit->second.state = MG_JOB_RUNNING;
    }
    v->in_use += need;
    v->queue.pop_front();
    v->active.push_back(j);
  }
  const uint32_t n = (uint32_t)v->active.size();
  if (n == 0) {
    v->last_frame_ms = (float)(1e3 * (wall_s() - t0));
    return MG_OK;
  }
  uint32_t stride = 0;
  uint64_t packed = 0;
  for (MgServerJob* j : v->active) {
    stride = std::max(stride, j->n_sub);
    packed += (uint64_t)j->sim->md.cap_impacts * j->n_sub;
  }
  int rc = server_reserve(v, n, packed);
  if (rc) return rc;
  size_t smem = 0;
  const float frame_dt = v->cfg.frame_dt;
  for (uint32_t k = 0; k < n; ++k) {
    MgServerJob* j = v->active[k];
    MgSim* s = j->sim;
    const MgSimulationParams& q = s->params.simulation;
    rc = fill_uniform(s, sim_drum(s), s->params.media, s->params.slurry, q.pbf_iterations, q.dem_iterations, 1, 1, 1);
    if (rc) return sfail(v, rc, "job %llu: %s", (unsigned long long)j->id, s->err.c_str());
    s->h_uni->fold_stress = 1u;
    std::memcpy(&v->h_uni[k], s->h_uni, sizeof(StepUniform));
    fill_desc(s);
    v->h_md[k] = s->md;
    v->h_md[k].out = v->d_out + (size_t)k * stride;
    v->h_md[k].stress_copy = v->d_stress + k;
    smem = std::max(smem, (size_t)s->md.smem_bytes);
    v->h_nsub[k] = j->n_sub;
    const float sub_dt = frame_dt / (float)j->n_sub;
    const float omega = mgh::mill_omega(s->params.mill);
    float angle = s->drum_angle;
    double now = s->sim_time;
    for (uint32_t t = 0; t < j->n_sub; ++t) {
      fill_angle(v->h_ang[(size_t)k * stride + t], angle, omega, sub_dt, now);
      angle = mgh::rem_euclid_r(angle + omega * sub_dt, mgh::TAU_F);
      now += (double)sub_dt;
    }
  }
  SCK(cudaMemcpyAsync(v->d_md, v->h_md, sizeof(MillDev) * n, cudaMemcpyHostToDevice, v->stream));
  SCK(cudaMemcpyAsync(v->d_uni, v->h_uni, sizeof(StepUniform) * n, cudaMemcpyHostToDevice, v->stream));
  SCK(cudaMemcpyAsync(v->d_ang, v->h_ang, sizeof(SubAngles) * n * stride, cudaMemcpyHostToDevice, v->stream));
  SCK(cudaMemcpyAsync(v->d_nsub, v->h_nsub, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, v->stream));
  // blocks run the jobs longest first (the last frame's device cycles; before their first frame,
  // sub-steps times particles)
  for (uint32_t k = 0; k < n; ++k) {
    MgServerJob* j = v->active[k];
    if (j->cost < 0.0) j->cost = (double)j->n_sub * ((double)j->sim->nf + 4.0 * (double)j->sim->nb);
    v->h_order[k] = k;
  }
  std::stable_sort(v->h_order, v->h_order + n,
                   [&](uint32_t x, uint32_t y) { return v->active[x]->cost > v->active[y]->cost; });
  SCK(cudaMemcpyAsync(v->d_order, v->h_order, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, v->stream));
  SCK(cudaEventRecord(v->ev0, v->stream));
  SCK(launch_substeps(v->d_md, n, v->d_uni, v->d_ang, stride, v->d_nsub, v->cfg.block_threads, smem, v->stream, 1,
                      v->d_order));
  SCK(cudaEventRecord(v->ev1, v->stream));
  SCK(cudaMemsetAsync(v->d_cursor, 0, sizeof(uint32_t), v->stream));
  SCK(launch_pack_impacts(v->d_md, n, v->d_nsub, v->d_packed, (uint32_t)std::min<uint64_t>(v->packed_cap, 0xFFFFFFF0ull),
                          v->d_cursor, v->d_table, v->stream));
  SCK(cudaMemcpyAsync(v->h_out, v->d_out, sizeof(StepOut) * n * stride, cudaMemcpyDeviceToHost, v->stream));
  SCK(cudaMemcpyAsync(v->h_table, v->d_table, sizeof(uint2) * n, cudaMemcpyDeviceToHost, v->stream));
  SCK(cudaMemcpyAsync(v->h_stress, v->d_stress, sizeof(StressState) * n, cudaMemcpyDeviceToHost, v->stream));
  SCK(cudaStreamSynchronize(v->stream));
  SCK(cudaEventElapsedTime(&v->last_kernel_ms, v->ev0, v->ev1));
  uint64_t total = 0;
  for (uint32_t k = 0; k < n; ++k) total = std::max<uint64_t>(total, (uint64_t)v->h_table[k].x + v->h_table[k].y);
  if (total > v->packed_cap) return sfail(v, MG_ERR_CAPACITY, "impact records exceed the server buffer");
  if (total)
    SCK(cudaMemcpyAsync(v->h_packed, v->d_packed, sizeof(MgImpactRecord) * total, cudaMemcpyDeviceToHost, v->stream));
  SCK(cudaStreamSynchronize(v->stream));
  v->frames += 1;
  const double t_end = wall_s();
  std::vector<uint32_t> failed(n, 0u);
  // the jobs' host folds are independent of one another: several host threads
  parallel_for(n, [&](uint32_t k) {
    MgServerJob* j = v->active[k];
    MgSim* s = j->sim;
    const uint32_t ns = j->n_sub;
    const StepOut* o = v->h_out + (size_t)k * stride;
    uint32_t e = 0;
    double cyc = 0.0;
    for (uint32_t t = 0; t < ns; ++t) {
      e |= o[t].err;
      for (int q = 0; q <= 14; ++q) cyc += (double)o[t].stage[q];
    }
    if (e) {
      failed[k] = 1u;
      return;
    }
    j->cost = cyc;
    s->stress = v->h_stress[k];
    std::memcpy(s->h_out, o, sizeof(StepOut) * ns);
    const MgImpactRecord* rec = v->h_packed + v->h_table[k].x;
    for (uint32_t t = 0; t < ns; ++t) {
      const uint32_t ni = std::min(o[t].n_impacts, s->md.cap_impacts);
      if (ni) std::memcpy(s->h_imp + (size_t)t * s->md.cap_impacts, rec, sizeof(MgImpactRecord) * ni);
      rec += ni;
    }
    s->max_disp = 0.0f;
    s->clamp_hits_frame = 0;
    const float sub_dt = frame_dt / (float)ns;
    const float omega = mgh::mill_omega(s->params.mill);
    for (uint32_t t = 0; t < ns; ++t) fold_substep(s, t, sub_dt, omega);
    s->last_fluid = o[ns - 1].fs;
    s->last_dem = o[ns - 1].ds;
    s->last_ctr = o[ns - 1].ctr;
    s->launches += 1;
  });
  std::vector<MgServerJob*> keep;
  keep.reserve(n);
  for (uint32_t k = 0; k < n; ++k) {
    MgServerJob* j = v->active[k];
    if (failed[k]) {
      retire(v, j, MG_JOB_FAILED);
      continue;
    }
    MgSim* s = j->sim;
    j->frames_done += 1;
    if (j->acc) seed_acc_observe(j->acc, s, j->frames_done);
    if (j->t_first < 0.0) j->t_first = t_end;
    if (j->frames_done >= j->frames_total) {
      retire(v, j, MG_JOB_FINISHED);
    } else {
      v->pending.push_back(job_update(j, MG_JOB_RUNNING));
      keep.push_back(j);
    }
  }
  v->active.swap(keep);
  v->last_frame_ms = (float)(1e3 * (wall_s() - t0));
  return MG_OK;
}

int mg_server_poll(MgServer* v, MgJobUpdate* out, uint32_t cap, uint32_t* n_out) {
  if (!v || (!out && cap)) return fail_global(MG_ERR_ARG, "null argument");
  const uint32_t n = (uint32_t)std::min<size_t>(cap, v->pending.size());
  if (n) std::memcpy(out, v->pending.data(), sizeof(MgJobUpdate) * n);
  v->pending.erase(v->pending.begin(), v->pending.begin() + n);
  if (n_out) *n_out = n;
  return MG_OK;
}

int mg_server_stats(MgServer* v, MgServerStats* out) {
  if (!v || !out) return fail_global(MG_ERR_ARG, "null argument");
  std::memset(out, 0, sizeof(*out));
  out->queued = (uint32_t)v->queue.size();
  out->active = (uint32_t)v->active.size();
  out->finished_total = v->finished_total;
  out->pending_updates = (uint32_t)v->pending.size();
  out->device_bytes_in_use = v->in_use;
  out->frames = v->frames;
  out->last_frame_ms = v->last_frame_ms;
  out->last_kernel_ms = v->last_kernel_ms;
  return MG_OK;
}

}  // extern "C"

// ====================================================================== grinding statistics
namespace {

const double THRESHOLDS_REL[6] = {0.03, 0.1, 0.3, 1.0, 3.0, 10.0};  // stress.rs:42

// StressAccum::metrics (stress.rs:186-237) with Simulation::metrics's arguments (lib.rs:383-390):
// the ball count, the 3D ball mass m3 = disc mass * 4/3 r, m3 g d and the EMA power draw.
MgStressMetrics stress_metrics_of(const MgSim* s) {
  const double r = (double)s->bmat.radius;
  const double m3 = (double)s->bmat.mass * 4.0 / 3.0 * r;
  const double d = 2.0 * r;
  const double scale_j = m3 * 9.81 * d;
  const StressState& st = s->stress;
  const double n = (double)std::max<uint32_t>(s->nb, 1u);
  const double power_draw_w = (double)s->power;
  MgStressMetrics o;
  std::memset(&o, 0, sizeof(o));
  for (int c = 0; c < 4; ++c) {
    o.impacts_per_ball_per_s[c] = (float)(st.count_rate[c] / n);
    if (st.count_rate[c] > 0.0) o.mean_se_scaled[c] = (float)(st.se_hat_rate[c] / st.count_rate[c]);
  }
  auto pooled = [&](int a, int b) {
    double w = st.count_rate[a] + st.count_rate[b];
    return w > 0.0 ? (float)((st.se_hat_rate[a] + st.se_hat_rate[b]) / w) : 0.0f;
  };
  const double total = stress_total_rate(st);
  const double power_per_ball = power_draw_w * d / n;
  o.ball_mass_3d_kg = (float)m3;
  o.scale_energy_j = (float)scale_j;
  o.impacts_total_per_ball_per_s = (float)(total / n);
  o.mean_se_scaled_drop = pooled(0, 2);
  o.mean_se_scaled_shear = pooled(1, 3);
  double se_sum = 0.0;
  for (int c = 0; c < 4; ++c) se_sum += st.se_hat_rate[c];
  o.stress_intensity_scaled = total > 0.0 ? (float)(se_sum / total) : 0.0f;
  o.wall_power_per_ball_w = (float)power_per_ball;
  o.specific_power_w_per_kg = (float)(power_per_ball / m3);
  for (int q = 0; q < 6; ++q) {
    o.thresholds_scaled[q] = (float)THRESHOLDS_REL[q];
    o.effective_power_per_ball_w[q] = (float)(st.above_rate_j[q] / n);
    o.cumulative_effective_energy_per_ball_j[q] = st.cum_above_j[q] / n;
  }
  o.cumulative_wall_energy_per_ball_j = st.cum_wall_j * d / n;
  o.cumulative_specific_energy_j_per_kg = st.cum_wall_j * d / n / m3;
  return o;
}

// batch.rs:126-139: the 16 per-frame scalars in name order
void seed_frame_values(const MgStressMetrics& m, double* v) {
  v[0] = m.specific_power_w_per_kg;
  v[1] = m.wall_power_per_ball_w;
  v[2] = m.impacts_total_per_ball_per_s;
  v[3] = m.mean_se_scaled_drop;
  v[4] = m.mean_se_scaled_shear;
  v[5] = m.stress_intensity_scaled;
  for (int c = 0; c < 4; ++c) v[6 + c] = m.impacts_per_ball_per_s[c];
  for (int q = 0; q < 6; ++q) v[10 + q] = m.effective_power_per_ball_w[q];
}

// batch.rs:141-159
double drift_per_rev_of(const double* y, size_t len, double frames_per_rev) {
  if (len < 2) return 0.0;
  const double n = (double)len;
  double sum = 0.0;
  for (size_t i = 0; i < len; ++i) sum += y[i];
  const double mean = sum / n, xm = (n - 1.0) / 2.0;
  double sxy = 0.0, sxx = 0.0;
  for (size_t i = 0; i < len; ++i) {
    sxy += ((double)i - xm) * (y[i] - mean);
    sxx += ((double)i - xm) * ((double)i - xm);
  }
  return std::fabs(mean) > 0.0 && sxx > 0.0 ? sxy / sxx * frames_per_rev / std::fabs(mean) : 0.0;
}

const char* const SEED_VALUE_NAMES[MG_SEED_VALUES] = {
    "specific_power_w_per_kg", "wall_power_per_ball_w", "impacts_total_per_ball_per_s", "mean_se_scaled_drop",
    "mean_se_scaled_shear", "stress_intensity_scaled", "impacts_per_ball_per_s.ball_ball_drop",
    "impacts_per_ball_per_s.ball_ball_shear", "impacts_per_ball_per_s.ball_wall_drop",
    "impacts_per_ball_per_s.ball_wall_shear", "effective_power_per_ball_w.thr0", "effective_power_per_ball_w.thr1",
    "effective_power_per_ball_w.thr2", "effective_power_per_ball_w.thr3", "effective_power_per_ball_w.thr4",
    "effective_power_per_ball_w.thr5", "window_specific_power_w_per_kg", "window_effective_power_per_ball_w.thr0",
    "window_effective_power_per_ball_w.thr1", "window_effective_power_per_ball_w.thr2",
    "window_effective_power_per_ball_w.thr3", "window_effective_power_per_ball_w.thr4",
    "window_effective_power_per_ball_w.thr5"};

}  // namespace

// batch::run_seed's window (batch.rs:40-107) of one seed, fed frame by frame: `warm` frames of
// warm-up, then `meas` measured frames whose stress scalars are averaged, with the window powers
// from the cumulative energies and the drift of the wall power per revolution.
struct SeedAcc {
  uint32_t warm = 0, meas = 0;
  double rev_s = 0.0;
  float k_cg = 1.0f;
  uint64_t seed = 0;
  MgStressMetrics start{};
  double sum[16] = {};
  std::vector<double> powers;
};

// Frames of run_seed's warm-up and measured windows (batch.rs:56-62); false when the mill speed
// or the revolutions are out of range.
bool seed_window(const MgParams& p, float warmup_revolutions, float measure_revolutions, uint32_t* warm,
                 uint32_t* meas, double* rev_s) {
  const double omega = (double)(mgh::mill_rpm(p.mill) * 2.0f * mgh::PI_F / 60.0f);
  if (omega <= 1e-6 || !(measure_revolutions >= 1.0f && warmup_revolutions >= 0.0f)) return false;
  *rev_s = 6.283185307179586 / omega;
  *warm = (uint32_t)std::round((double)warmup_revolutions * *rev_s * 60.0);
  *meas = (uint32_t)std::max(std::round((double)measure_revolutions * *rev_s * 60.0), 1.0);
  return true;
}

SeedAcc* seed_acc_new(const MgParams& p, uint32_t warm, uint32_t meas, double rev_s) {
  SeedAcc* a = new SeedAcc();
  a->warm = warm;
  a->meas = meas;
  a->rev_s = rev_s;
  a->seed = p.simulation.seed;
  a->k_cg = mgh::effective_media(p).scale_factor;
  a->powers.assign(meas, 0.0);
  return a;
}
void seed_acc_free(SeedAcc* a) { delete a; }
// Called with the initial state (frames_done 0) and after every frame.
void seed_acc_observe(SeedAcc* a, const MgSim* s, uint32_t frames_done) {
  if (frames_done == a->warm) a->start = stress_metrics_of(s);
  if (frames_done <= a->warm || frames_done > a->warm + a->meas) return;
  const MgStressMetrics m = stress_metrics_of(s);
  double v[16];
  seed_frame_values(m, v);
  for (int k = 0; k < 16; ++k) a->sum[k] += v[k];
  a->powers[frames_done - a->warm - 1] = (double)m.wall_power_per_ball_w;
}
// The seed's result once its last measured frame has been observed.
void seed_acc_finish(const SeedAcc* a, const MgSim* s, MgSeedResult* r) {
  const MgStressMetrics end = stress_metrics_of(s);
  const double n = (double)a->meas, window_s = n * (double)(1.0f / 60.0f);
  std::memset(r, 0, sizeof(*r));
  r->seed = a->seed;
  r->window_s = window_s;
  r->coarse_graining_factor = a->k_cg;
  for (int k = 0; k < 16; ++k) r->values[k] = a->sum[k] / n;
  r->values[16] = (end.cumulative_specific_energy_j_per_kg - a->start.cumulative_specific_energy_j_per_kg) / window_s;
  for (int q = 0; q < 6; ++q)
    r->values[17 + q] =
        (end.cumulative_effective_energy_per_ball_j[q] - a->start.cumulative_effective_energy_per_ball_j[q]) /
        window_s;
  r->power_drift_rel_per_rev = drift_per_rev_of(a->powers.data(), a->meas, a->rev_s * 60.0);
}

extern "C" {

int mg_stress_metrics(MgSim* s, MgStressMetrics* out) {
  if (!s || !out) return fail_global(MG_ERR_ARG, "null argument");
  *out = stress_metrics_of(s);
  return MG_OK;
}

const char* mg_seed_value_name(uint32_t k) { return k < MG_SEED_VALUES ? SEED_VALUE_NAMES[k] : ""; }

// batch::run_seed for every seed at once: the seeds are the mills of one batch, so every frame of
// the sweep is one launch; per seed the frames, statistics and sums are those of run_seed alone.
int mg_seed_sweep(const MgParams* params, const uint64_t* seeds, uint32_t n_seeds, float warmup_revolutions,
                  float measure_revolutions, MgSeedResult* out) {
  if (!params || n_seeds == 0 || !seeds || !out) return fail_global(MG_ERR_ARG, "null argument or no seeds");
  uint32_t warm = 0, meas = 0;
  double rev_s = 0.0;
  if (!seed_window(*params, warmup_revolutions, measure_revolutions, &warm, &meas, &rev_s))
    return fail_global(MG_ERR_ARG, "mill speed must be > 0, measure_revolutions >= 1 and warmup_revolutions >= 0");
  const float frame_s = 1.0f / 60.0f;
  std::vector<MgParams> ps(n_seeds, *params);
  for (uint32_t i = 0; i < n_seeds; ++i) ps[i].simulation.seed = seeds[i];
  MgBatch* b = nullptr;
  int rc = mg_batch_create(ps.data(), n_seeds, &b);
  if (rc) return rc;
  std::vector<SeedAcc*> acc(n_seeds);
  for (uint32_t i = 0; i < n_seeds; ++i) acc[i] = seed_acc_new(ps[i], warm, meas, rev_s);
  if (warm) rc = mg_batch_step_frames(b, warm, frame_s);
  for (uint32_t i = 0; i < n_seeds && !rc; ++i) seed_acc_observe(acc[i], b->mills[i], warm);
  for (uint32_t f = 0; f < meas && !rc; ++f) {
    rc = mg_batch_step_frames(b, 1, frame_s);
    for (uint32_t i = 0; i < n_seeds && !rc; ++i) seed_acc_observe(acc[i], b->mills[i], warm + f + 1);
  }
  if (!rc)
    for (uint32_t i = 0; i < n_seeds; ++i) seed_acc_finish(acc[i], b->mills[i], &out[i]);
  for (SeedAcc* a : acc) seed_acc_free(a);
  if (rc) {
    std::string e = b->err;
    mg_batch_destroy(b);
    return fail_global(rc, "%s", e.c_str());
  }
  mg_batch_destroy(b);
  return MG_OK;
}

// batch.rs:161-190 combine
int mg_seed_combine(const MgSeedResult* r, uint32_t n, double* mean, double* std_err) {
  if (n == 0) return fail_global(MG_ERR_ARG, "no results to combine");
  if (!r || !mean || !std_err) return fail_global(MG_ERR_ARG, "null argument");
  const double nn = (double)n;
  for (int k = 0; k < MG_SEED_VALUES; ++k) {
    double s = 0.0;
    for (uint32_t i = 0; i < n; ++i) s += r[i].values[k];
    const double m = s / nn;
    double se = 0.0;
    if (n >= 2) {
      double v = 0.0;
      for (uint32_t i = 0; i < n; ++i) {
        double dv = r[i].values[k] - m;
        v += dv * dv;
      }
      se = std::sqrt(v / (nn - 1.0) / nn);
    }
    mean[k] = m;
    std_err[k] = se;
  }
  return MG_OK;
}

double mg_seed_drift_per_rev(const double* y, uint32_t n, double frames_per_rev) {
  return y ? drift_per_rev_of(y, n, frames_per_rev) : 0.0;
}

}  // extern "C"
