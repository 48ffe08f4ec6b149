// fdtd_batch.cuh -- batched step kernels: many independent problems of uneven
// size advance together, one launch per kernel kind per step for the whole
// batch.  Each problem (instance) keeps its own device state and parameter
// block; the H and E launches walk one flat list of tiles across all
// instances (either one block per tile, or a persistent grid that claims runs
// of consecutive tiles from a counter), and the mid and epilogue launches map
// blocks to instances through a per-block table.
#pragma once
#include "fdtd_common.cuh"
#include "fdtd_step.cuh"

namespace fdtd {

// One instance of a batch: the parameter blocks of its four kernels.
template <typename T, class C>
struct Instance {
  StepParams<T, C> sp;
  Probes pr;
  FarField ff;
};

// A tile of one instance: the (blockIdx.x, blockIdx.y, blockIdx.z) it would
// have in that instance's own H/E launch.
struct BatchTile {
  unsigned short inst, bx, by, bz;
};

// Mid/epilogue block -> (instance, block index inside that instance's launch).
struct BatchBlock {
  int inst, local;
};

// Shared state of a batch on the device.
struct BatchCtl {
  int ts;          // step counter shared by every instance
  int next[2];     // tile counters of the persistent H (0) and E (1) launches
};

// Copies a parameter block (global) into shared memory with 8-byte words.
template <class P>
__device__ __forceinline__ void load_block_params(P* dst, const P* src) {
  static_assert(sizeof(P) % 8 == 0, "parameter block must be 8-byte sized");
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int w = tid; w < (int)(sizeof(P) / 8); w += nt) d[w] = __ldg(s + w);
}

// H (ELECTRIC=false) or E (true) update over the batch's tiles.  PERSIST: a
// persistent grid whose blocks claim `group` consecutive tiles at a time;
// otherwise one block per tile.  A block copies its member's parameter block
// into shared memory: reading it in place from global memory costs more (the
// loads are repeated after every field store, which may alias them, and what
// the compiler keeps in registers spills).
template <typename T, class C, bool EXACT, int PF, bool ELECTRIC, bool PERSIST>
__global__ void __launch_bounds__(256, MinBlocks<T, PF>::value)
    k_batch_half(const Instance<T, C>* __restrict__ inst, const BatchTile* __restrict__ tiles, int ntiles,
                 BatchCtl* ctl, int group) {
  __shared__ __align__(16) unsigned char raw[sizeof(StepParams<T, C>)];
  __shared__ int s_claim;
  StepParams<T, C>* sp = reinterpret_cast<StepParams<T, C>*>(raw);
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  if (!ELECTRIC && blockIdx.x == 0 && lead) ctl->ts += 1;  // first kernel of a step advances the counter
  if constexpr (!PERSIST) {
    const BatchTile t = tiles[blockIdx.x];
    load_block_params(sp, &inst[t.inst].sp);
    __syncthreads();
    if (ELECTRIC)
      step_e_tile<T, C, EXACT, PF>(*sp, t.bx, t.by, t.bz);
    else
      step_h_tile<T, C, EXACT, PF>(*sp, t.bx, t.by, t.bz);
  } else {
    int cur = -1;
    for (;;) {
      if (lead) s_claim = atomicAdd(&ctl->next[ELECTRIC ? 1 : 0], group);
      __syncthreads();
      const int first = s_claim;
      if (first >= ntiles) break;
      const int last = min(first + group, ntiles);
      for (int q = first; q < last; q++) {
        const BatchTile t = tiles[q];
        if (t.inst != cur) {
          __syncthreads();  // every thread is done with the previous block
          load_block_params(sp, &inst[t.inst].sp);
          cur = t.inst;
          __syncthreads();
        }
        if (ELECTRIC)
          step_e_tile<T, C, EXACT, PF>(*sp, t.bx, t.by, t.bz);
        else
          step_h_tile<T, C, EXACT, PF>(*sp, t.bx, t.by, t.bz);
      }
      __syncthreads();  // s_claim is rewritten by the next claim
    }
  }
}

// Grouped mode: up to kGroupMembers members' parameter blocks travel as ONE
// kernel parameter (__grid_constant__, the constant bank), so the tile code
// reads them as it reads a single problem's parameters: no copy into shared
// memory, and no reload after every field store, since no store can alias
// the constant bank.  A launch covers its members' tiles back to back:
// member m owns blocks [first[m], first[m+1]) and lays them out as its own
// (gx x gy x gz) launch would, x fastest.
constexpr int kGroupMembers = 22;  // 22 blocks of at most 1.4 KB + tables: inside the 32 KB parameter limit

template <typename T, class C>
struct BatchGroup {
  int n;                         // members in this launch
  int* ts;                       // H launch of the step's first group: advances the shared step counter
  int first[kGroupMembers + 1];  // first block of each member, and the block count at n
  int gx[kGroupMembers], gy[kGroupMembers];
  StepParams<T, C> sp[kGroupMembers];
};

template <typename T, class C, bool EXACT, int PF, bool ELECTRIC>
__global__ void __launch_bounds__(256, MinBlocks<T, PF>::value)
    k_batch_group(const __grid_constant__ BatchGroup<T, C> g) {
  const int b = blockIdx.x;
  if (!ELECTRIC && g.ts && b == 0 && threadIdx.x == 0 && threadIdx.y == 0) *g.ts += 1;
  // the member that owns this block: every operand is uniform over the block
  int m = 0;
#pragma unroll 1
  while (m + 1 < g.n && b >= g.first[m + 1]) m++;
  const int local = b - g.first[m];
  const int gx = g.gx[m], gy = g.gy[m];
  const int bx = local % gx, r = local / gx;
  const int by = r % gy, bz = r / gy;
  if (ELECTRIC)
    step_e_tile<T, C, EXACT, PF>(g.sp[m], bx, by, bz);
  else
    step_h_tile<T, C, EXACT, PF>(g.sp[m], bx, by, bz);
}

// Ex(i=0) scratch planes and port currents of every instance.  Also re-arms
// the persistent tile counters: the H launch before this one is complete and
// the E launch after it has not started.
template <typename T, class C, bool EXACT>
__global__ void __launch_bounds__(256)
    k_batch_mid(const Instance<T, C>* __restrict__ inst, const BatchBlock* __restrict__ blocks, BatchCtl* ctl,
                int ninst) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->next[0] = 0;
    ctl->next[1] = 0;
    // time-blocked DFT: at a block boundary the previous block has been flushed
    const int ts = ctl->ts;
    for (int q = 0; q < ninst; q++)
      if (inst[q].sp.dft_block > 0 && ts % inst[q].sp.dft_block == 0) *inst[q].sp.dft_done = ts;
  }
  const BatchBlock b = blocks[blockIdx.x];
  const Instance<T, C>& in = inst[b.inst];
  step_mid_thread<T, C, EXACT>(in.sp, in.pr, (long long)b.local * blockDim.x + threadIdx.x);
}

// Far-field DFT and port voltages of every instance.
template <typename T, class C>
__global__ void __launch_bounds__(256)
    k_batch_epilogue(const Instance<T, C>* __restrict__ inst, const BatchBlock* __restrict__ blocks) {
  const BatchBlock b = blocks[blockIdx.x];
  const Instance<T, C>& in = inst[b.inst];
  epilogue_thread<T>(in.sp.f, in.sp.g, in.ff, in.pr, in.sp.ts, (long long)b.local * blockDim.x + threadIdx.x);
}

// Time-blocked DFT flush of every member (see k_dft_flush).
template <typename T, class C>
__global__ void __launch_bounds__(256)
    k_batch_flush(const Instance<T, C>* __restrict__ inst, const BatchBlock* __restrict__ blocks, int upto) {
  const BatchBlock b = blocks[blockIdx.x];
  const Instance<T, C>& in = inst[b.inst];
  dft_flush_thread(in.ff, in.sp.ts, upto, (long long)b.local * blockDim.x + threadIdx.x);
}

}  // namespace fdtd
