// Helper blocks of a single-mill launch. A mill's sub-step is one thread block's work, but a few
// stages loop over the balls with one warp per ball and nothing shared between balls; in a
// single-mill launch those loops are spread over the warps of the mill's block and of helper
// blocks (a cooperative launch, so all blocks are resident). The mill's block publishes each such
// phase in the control block (after its own writes that the phase reads), runs its share, and
// waits until every helper block has finished its share; the helper blocks loop on the control
// block until the mill's block publishes WIDE_EXIT. Every wait is bounded: after about ten seconds
// it sets ERR_WIDE and gives up, so a block that stops answering ends the launch with an error.
// Memory ordering follows the usual grid-barrier pattern: writes, block barrier, thread 0's
// device-scope fence, then the flag; on the other side the flag, thread 0's fence, block barrier.
#pragma once

#include "mill_block.cuh"

namespace mg {

enum : uint32_t {
  WIDE_EXIT = 0,
  WIDE_ADHESION = 1,
  WIDE_GROUPS = 2,
  WIDE_LINKS = 3,
  WIDE_DRAG_ITEMS = 4,
  WIDE_BUOYANCY_ITEMS = 5,
  WIDE_CG_SETUP = 6,
  WIDE_JOINT_APPLY = 7,
  WIDE_DRAG_PRE = 8,
  WIDE_FLUID_PREP = 9,
  WIDE_BESIDE_DRAG = 10,
  WIDE_DRAG_LISTS = 11
};


__shared__ uint32_t g_wide_seq;  // phases the mill's block has published in this launch

// Waits (thread 0) until *p >= target; false when `limit` clock cycles ran out first.
__device__ inline bool wide_wait(const uint32_t* p, uint32_t target, long long limit = WIDE_TIMEOUT_CYCLES) {
  const long long t0 = clock64();
  while ((int32_t)(*reinterpret_cast<const volatile uint32_t*>(p) - target) < 0) {
    if (clock64() - t0 > limit) return false;
    __nanosleep(64);
  }
  return true;
}

// Mill block (helpers > 0): publishes a phase after the block's writes that it reads. pre(c), run
// by thread 0 before the flag, fills the phase's own fields of the control block.
template <class Pre>
__device__ void wide_publish(const MillDev& m, uint32_t phase, const GridHdr* hdr, const float2* vin, float2* vout,
                             Pre pre) {
  __syncthreads();
  WideCtl* c = m.wide;
  if (tid() == 0) {
    if (hdr) c->hdr = *hdr;
    c->vin = vin;
    c->vout = vout;
    c->phase = phase;
    c->counter = 0;
    pre(c);
    g_wide_seq += 1;
    __threadfence();
    *reinterpret_cast<volatile uint32_t*>(&c->seq) = g_wide_seq;
  }
}

// Mill block (helpers > 0): waits until every helper block has finished the last published phase;
// afterwards the block reads what they wrote.
__device__ inline void wide_finish(const MillDev& m) {
  __syncthreads();
  if (tid() == 0) {
    WideCtl* c = m.wide;
    const long long lim = m.wide_wait_cycles > 0 ? m.wide_wait_cycles : WIDE_TIMEOUT_CYCLES;
    if (!wide_wait(&c->done, g_wide_seq * (m.helpers + m.test_extra_helpers), lim)) {
      atomicOr(m.err, ERR_WIDE);
      // the helper blocks that did answer finish this phase before the mill's block goes on and
      // overwrites what they read (bounded too); the launch then ends at the next error check
      wide_wait(&c->done, g_wide_seq * m.helpers);
    }
    __threadfence();
  }
  __syncthreads();
}

// Mill block: one phase over all of the mill's warps. share(w0, nw) is called by every thread of
// the block with w0 = the thread's warp and nw = the warps of all of the mill's blocks.
template <class F>
__device__ void wide_phase(const MillDev& m, uint32_t phase, const GridHdr* hdr, const float2* vin, float2* vout,
                           F share) {
  const uint32_t warp = tid() >> 5, nwarps = nthr() >> 5;
  if (m.helpers == 0) {
    share(warp, nwarps);
    __syncthreads();
    return;
  }
  wide_publish(m, phase, hdr, vin, vout, [](WideCtl*) {});
  share(warp, (1u + m.helpers) * nwarps);
  wide_finish(m);
}

template <class F>
__device__ void wide_phase(const MillDev& m, uint32_t phase, const GridHdr* hdr, F share) {
  wide_phase(m, phase, hdr, nullptr, nullptr, share);
}

// Mill block: the helper blocks' count of the last phase (call after wide_phase).
__device__ inline uint32_t wide_counter(const MillDev& m) {
  return m.helpers ? *reinterpret_cast<const volatile uint32_t*>(&m.wide->counter) : 0u;
}

// Mill block, at the end of the launch: releases the helper blocks.
__device__ inline void wide_exit(const MillDev& m) {
  if (m.helpers == 0) return;
  __syncthreads();
  if (tid() == 0) {
    WideCtl* c = m.wide;
    c->phase = WIDE_EXIT;
    g_wide_seq += 1;
    __threadfence();
    *reinterpret_cast<volatile uint32_t*>(&c->seq) = g_wide_seq;
  }
}

// Helper block: runs its share of every published phase until WIDE_EXIT. run(phase, hdr, vin,
// vout, w0, nw) returns the thread's part of the phase's count.
template <class Run>
__device__ void wide_helper(const MillDev& m, Run run) {
  __shared__ uint32_t ph;
  __shared__ GridHdr hdr;
  __shared__ const float2* vin;
  __shared__ float2* vout;
  WideCtl* c = m.wide;
  const uint32_t nwarps = nthr() >> 5;
  const uint32_t w0 = blockIdx.x * nwarps + (tid() >> 5), nw = (1u + m.helpers) * nwarps;
  for (uint32_t seq = 1;; ++seq) {
    if (tid() == 0) {
      if (!wide_wait(&c->seq, seq)) {
        atomicOr(m.err, ERR_WIDE);
        ph = WIDE_EXIT;
      } else {
        __threadfence();
        ph = *reinterpret_cast<const volatile uint32_t*>(&c->phase);
        hdr = c->hdr;
        vin = c->vin;
        vout = c->vout;
      }
    }
    __syncthreads();
    const uint32_t p = ph;
    if (p == WIDE_EXIT) return;
    const uint32_t part = block_sum_u(run(p, hdr, vin, vout, w0, nw));
    if (tid() == 0) {
      if (part) atomicAdd(&c->counter, part);
      __threadfence();
      atomicAdd(&c->done, 1u);
    }
  }
}

}  // namespace mg
