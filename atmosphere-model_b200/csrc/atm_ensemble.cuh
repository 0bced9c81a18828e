// Persistent ensemble kernel of the mixed form: many independent dycore
// domains (members of uneven sizes) advanced by a whole run of steps in ONE
// cooperative launch.
//
// Every step of every member is the single-domain sequence of stages
// (src/mod_model.f90:146-177): C-grid mass sweep, C-grid column, C-grid
// momentum sweep, C-grid halo fill, D-grid ring copy, D-grid mass sweep,
// D-grid column, corner interpolation, D-grid momentum sweep, [ring copy,
// wind remap, energy remap], D-grid halo fill.  A stage's work is a queue
// of warp-sized items over all members -- a (member, layer, strip) of a
// marching sweep, 32 consecutive columns or corners, or 8 x 32 ring points
// of a level -- which the resident warps take in turn, so small and large
// members share the GPU within each stage.  Two schedules:
//  * barrier (default): every member takes a stage together, and stages are
//    separated by a grid-wide barrier whose wait is bounded: a block that
//    waits longer than the plan's limit raises the error word and returns,
//    and every other block returns at its next barrier or as soon as it
//    sees the error, so a failed barrier ends the launch instead of hanging
//    it;
//  * dataflow: no grid barrier; each member advances through its stages on
//    its own (ens_dataflow), so the stages of different members overlap.
//
// The per-member strip height of the marching sweeps (16, 32 or 64 rows)
// comes from the plan (an autotuned table keyed on the member's grid size).
// Fields written by one stage are read by later stages of the same launch,
// so every stage reads with plain (coherent) loads, never through the
// read-only data path; the fences of the barrier (or of the dataflow
// tickets) order the writes before them.
// The stage bodies are the single-domain kernels' device functions, so a
// member's results are bit-identical to stepping it alone.
#pragma once

#include "atm_kernels.cuh"
#include "atm_march.cuh"

namespace atm {

// a member as the persistent kernel sees it
struct EnsMember {
  Geom g;
  Consts cc, cd;  // the C-grid half step's (dt/2) and the D-grid step's (dt) constants
  RemapArgs ra;
  void* st[2][4];  // the two time levels of dp, pt, ud, vd
  void* cg[4];     // dpc, ptc, uc, vc
  double *pkap, *gz, *pkapb, *gzb;
  void *urem, *vrem;
  Status* status;
  int cur0;  // time level holding the state at launch
  int tys;   // strip height of its marching sweeps: 16, 32 or 64
};

enum EnsStage {
  E_CMASS, E_CCOL, E_CMOM, E_CHALO, E_DRING, E_DMASS, E_DCOL, E_DCORN, E_DMOM, E_RRING, E_RWIND, E_RENER, E_DHALO,
  E_NSTAGE
};

struct EnsPlan {
  const EnsMember* m;
  const long long* off;  // [E_NSTAGE][nm + 1]: prefix sums of the members' items
  int nm, nsteps, remap_every;
  unsigned* bar;         // arrival count, generation
  unsigned expect;       // blocks a barrier waits for (the grid; one more makes every barrier run out)
  int* err;              // raised when a barrier wait ran out
  long long timeout_ns;  // limit of one barrier wait
  unsigned long long* stage_ns;  // optional: nanoseconds between barrier exits, summed per stage (block 0's clock)
  // dataflow schedule (used when dataflow != 0): per member, the phase
  // ticket (phase << 32 | next item to claim) and the items done in the
  // phase; the count of members that finished the launch
  int dataflow;
  unsigned long long* tk;
  unsigned* dn;
  unsigned* fin;
};

__host__ __device__ inline long long ens_div_up(long long a, long long b) { return (a + b - 1) / b; }

// strips of a marching sweep over [lo, n-1+hi]^2
__host__ __device__ inline void ens_strips(const Geom& g, int lo, int hi, int tys, int& sxn, int& syn) {
  sxn = (int)ens_div_up(g.nx - lo + hi, MOUT);
  syn = (int)ens_div_up(g.ny - lo + hi, tys);
}
// ring points of one level and field in a warp item: ENS_RING_R per lane
constexpr int ENS_RING_R = 8;
__host__ __device__ inline int ens_ring_chunks(const Geom& g) {
  return (int)ens_div_up(2 * H * (g.nx + 2 * H) + 2 * H * g.ny, 32 * ENS_RING_R);
}

// warp items of a member in a stage
__host__ __device__ inline long long ens_items(const Geom& g, int stage, int tys) {
  int sxn = 0, syn = 0;
  switch (stage) {
    case E_CMASS: ens_strips(g, -2, 2, tys, sxn, syn); return (long long)sxn * syn * g.L;
    case E_DMASS: ens_strips(g, -3, 3, tys, sxn, syn); return (long long)sxn * syn * g.L;
    case E_CMOM:
    case E_DMOM: ens_strips(g, 0, 0, tys, sxn, syn); return (long long)sxn * syn * g.L;
    case E_CCOL:
    case E_DCOL: return ens_div_up((long long)(g.nx + 4) * (g.ny + 4), 32);
    case E_DCORN: return ens_div_up((long long)(g.nx + 1) * (g.ny + 1), 32);
    case E_CHALO:
    case E_DRING:
    case E_RRING:
    case E_DHALO: return (long long)ens_ring_chunks(g) * g.L * 4;
    case E_RWIND: return ens_div_up(2LL * (g.nx + 2) * (g.ny + 2), 32);
    case E_RENER: return ens_div_up((long long)g.nx * g.ny, 32);
    default: return 0;
  }
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier with a bounded wait; false in every thread of the block
// when this or an earlier barrier failed.
__device__ __forceinline__ bool ens_barrier(const EnsPlan& p) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = p.bar + 1;
    const unsigned g0 = *gen;
    __threadfence();
    bool ok = true;
    if (atomicAdd(p.bar, 1u) + 1 == p.expect) {
      atomicExch(p.bar, 0u);
      __threadfence();
      atomicAdd(p.bar + 1, 1u);
    } else {
      const long long t0 = global_ns();
      while (*gen == g0) {
        if (*(volatile int*)p.err != 0) {  // another block's wait ran out: leave at once
          ok = false;
          break;
        }
        if (global_ns() - t0 > p.timeout_ns) {
          ok = false;
          atomicOr(p.err, 1);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    s_ok = ok && *(volatile int*)p.err == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// the member of a stage's item (binary search of the prefix sums)
__device__ __forceinline__ int ens_member(const long long* off, int nm, long long item) {
  int lo = 0, hi = nm - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// one strip item of a marching sweep at the member's strip height
template <int TYS, typename F>
__device__ __forceinline__ void ens_strip_item(const Geom& g, int lo, int hi, long long li, F&& body) {
  int sxn, syn;
  ens_strips(g, lo, hi, TYS, sxn, syn);
  const int sx = (int)(li % sxn);
  const int sy = (int)((li / sxn) % syn);
  const int k = (int)(li / ((long long)sxn * syn));
  body(sx, sy, k);
}

// The stage bodies are not inlined: each keeps the register allocation of
// its single-domain kernel instead of the union of all of them.
template <typename T, typename S, typename C, int TYS>
__device__ __noinline__ void ens_cmass(const EnsMember& M, int cur, long long li) {
  ens_strip_item<TYS>(M.g, -2, 2, li, [&](int sx, int sy, int k) {
    void* const* so = M.st[cur];
    mass_strip<T, TYS, true, S, C, false>(M.g, M.cc, (const S*)so[0], (const S*)so[1], (const S*)so[2], (const S*)so[3],
                                   nullptr, (C*)M.cg[0], (C*)M.cg[1], -2, 2, nullptr, sx, sy, k);
  });
}
template <typename T, typename S, typename C, int TYS>
__device__ __noinline__ void ens_cmom(const EnsMember& M, int cur, long long li) {
  ens_strip_item<TYS>(M.g, 0, 0, li, [&](int sx, int sy, int k) {
    void* const* so = M.st[cur];
    c_mom_strip<T, TYS, S, C, false>(M.g, M.cc, (const S*)so[2], (const S*)so[3], M.pkap, M.gz, (C*)M.cg[2], (C*)M.cg[3],
                              sx, sy, k);
  });
}
template <typename T, typename S, typename C, int TYS>
__device__ __noinline__ void ens_dmass(const EnsMember& M, int cur, long long li) {
  ens_strip_item<TYS>(M.g, -3, 3, li, [&](int sx, int sy, int k) {
    void* const* so = M.st[cur];
    void* const* sn = M.st[cur ^ 1];
    mass_strip<T, TYS, false, S, C, false>(M.g, M.cd, (const S*)so[0], (const S*)so[1], (const C*)M.cg[2], (const C*)M.cg[3],
                                    nullptr, (S*)sn[0], (S*)sn[1], -3, 3, &M.status->nonfinite_step, sx, sy, k);
  });
}
template <typename T, typename S, typename C, int TYS>
__device__ __noinline__ void ens_dmom(const EnsMember& M, int cur, long long li) {
  ens_strip_item<TYS>(M.g, 0, 0, li, [&](int sx, int sy, int k) {
    void* const* so = M.st[cur];
    void* const* sn = M.st[cur ^ 1];
    d_mom_strip<T, TYS, S, C, false>(M.g, M.cd, (const S*)so[2], (const S*)so[3], (const C*)M.cg[2], (const C*)M.cg[3],
                              M.pkapb, M.gzb, (S*)sn[2], (S*)sn[3], &M.status->nonfinite_step, sx, sy, k);
  });
}

template <typename T, typename S, typename C, int TYS>
__device__ __forceinline__ void ens_sweep(int stage, const EnsMember& M, int cur, long long li) {
  if (stage == E_CMASS) ens_cmass<T, S, C, TYS>(M, cur, li);
  else if (stage == E_CMOM) ens_cmom<T, S, C, TYS>(M, cur, li);
  else if (stage == E_DMASS) ens_dmass<T, S, C, TYS>(M, cur, li);
  else ens_dmom<T, S, C, TYS>(M, cur, li);
}

template <typename S, int LM>
__device__ __noinline__ void ens_rwind(const EnsMember& M, int src, long long idx) {
  const Geom& g = M.g;
  void* const* s = M.st[src];
  const long long wh = (long long)(g.nx + 2) * (g.ny + 2);
  if (idx >= 2 * wh) return;
  remap_winds_at<S, LM, float>(g, M.ra, (const S*)s[0], (const S*)s[2], (const S*)s[3], (S*)M.urem, (S*)M.vrem, nullptr,
                        M.status, (int)(idx % wh), (int)(idx / wh));
}
template <typename S, int LM>
__device__ __noinline__ void ens_rener(const EnsMember& M, int src, long long idx) {
  void* const* s = M.st[src];
  void* const* d = M.st[src ^ 1];
  // the persistent kernel serves the mixed form only (atm_ensemble_create)
  remap_energy_at<S, LM, DevicePow>(M.g, M.ra, (const S*)s[0], (const S*)s[1], (const S*)s[2], (const S*)s[3],
                                    (const S*)M.urem, (const S*)M.vrem, M.gz, (S*)d[0], (S*)d[1], (S*)d[2], (S*)d[3],
                                    nullptr, M.status, (int)idx);
}
template <typename S, int LM>
__device__ __forceinline__ void ens_remap(int stage, const EnsMember& M, int src, long long idx) {
  if (stage == E_RWIND) ens_rwind<S, LM>(M, src, idx);
  else ens_rener<S, LM>(M, src, idx);
}

template <typename T, typename S, typename C>
__device__ __forceinline__ void ens_item(int stage, const EnsMember& M, int cur, long long li) {
  const Geom& g = M.g;
  const int lane = threadIdx.x & 31;
  switch (stage) {
    case E_CMASS:
    case E_CMOM:
    case E_DMASS:
    case E_DMOM:
      if (M.tys == 16) ens_sweep<T, S, C, 16>(stage, M, cur, li);
      else if (M.tys == 32) ens_sweep<T, S, C, 32>(stage, M, cur, li);
      else ens_sweep<T, S, C, 64>(stage, M, cur, li);
      break;
    case E_CCOL:
      column_at<C, FormPow<T>>(g, M.cc, (const C*)M.cg[0], (const C*)M.cg[1], M.pkap, M.gz, -2, 2, nullptr,
                   (int)(li * 32 + lane));
      break;
    case E_DCOL: {
      void* const* sn = M.st[cur ^ 1];
      column_at<S, FormPow<T>>(g, M.cd, (const S*)sn[0], (const S*)sn[1], M.pkap, M.gz, -2, 2, nullptr, (int)(li * 32 + lane));
      break;
    }
    case E_DCORN:
      corner_at<4>(g, M.pkap, M.gz, M.pkapb, M.gzb, 1, 0, g.L, (int)(li * 32 + lane));
      break;
    case E_CHALO:
    case E_DRING:
    case E_RRING:
    case E_DHALO: {
      const int chunks = ens_ring_chunks(g);
      const int idx = (int)(li % chunks) * 32 * ENS_RING_R + lane;
      const int k = (int)((li / chunks) % g.L);
      const int f = (int)(li / ((long long)chunks * g.L));
      if (stage == E_CHALO) ring_batch<C, false, ENS_RING_R>(g, (C*)M.cg[f], nullptr, idx, k);
      else if (stage == E_DHALO) ring_batch<S, false, ENS_RING_R>(g, (S*)M.st[cur][f], nullptr, idx, k);
      else ring_batch<S, true, ENS_RING_R>(g, (S*)M.st[cur ^ 1][f], (const S*)M.st[cur][f], idx, k);  // new level keeps the old ring
      break;
    }
    case E_RWIND:
    case E_RENER:
      if (g.L <= 32) ens_remap<S, 32>(stage, M, cur, li * 32 + lane);
      else ens_remap<S, 64>(stage, M, cur, li * 32 + lane);  // members hold at most 64 layers
      break;
    default:
      break;
  }
}

// Phase ph of a launch (the stages of all steps in order, 10 per step and 13
// on a remap step): its stage and the parity of the time-level swaps before
// it (a swap follows the D-grid momentum sweep and the energy remap).
__device__ __forceinline__ void ens_phase(int ph, int R, int& stage, int& flip) {
  constexpr int kStep[10] = {E_CMASS, E_CCOL, E_CMOM, E_CHALO, E_DRING, E_DMASS, E_DCOL, E_DCORN, E_DMOM, E_DHALO};
  if (R <= 0) {
    const int s = ph / 10, j = ph - 10 * (ph / 10);
    stage = kStep[j];
    flip = (s + (j == 9 ? 1 : 0)) & 1;
    return;
  }
  const int per = 10 * R + 3;  // phases of a remap cycle
  const int c = ph / per, q = ph - per * c;
  const int base = c * (R + 1);  // swaps of the earlier cycles
  if (q < 10 * (R - 1)) {
    const int s = q / 10, j = q - 10 * s;
    stage = kStep[j];
    flip = (base + s + (j == 9 ? 1 : 0)) & 1;
  } else {
    const int j = q - 10 * (R - 1);  // the remap step: all 13 stages in order
    stage = j;
    flip = (base + (R - 1) + (j > E_DMOM ? 1 : 0) + (j > E_RENER ? 1 : 0)) & 1;
  }
}

__device__ __forceinline__ long long ens_count(const EnsPlan& p, int stage, int m) {
  const long long* off = p.off + (long long)stage * (p.nm + 1);
  return off[m + 1] - off[m];
}

// Dataflow schedule: no grid barrier.  Each member advances through its
// phases on its own: a warp claims the next item of any member whose
// current phase has items left (an atomic add on the member's ticket), runs
// it, and the warp completing a phase's last item opens the member's next
// phase.  So the compute-bound sweeps of some members overlap the
// memory-bound column, corner, ring and remap passes of others.  Writes of
// a phase are released by a fence before its completion count and acquired
// by a fence after the claim of a later phase's item.  A warp that finds
// no work for longer than the plan's limit raises the error word and
// leaves; the others leave at their next idle check.
template <typename T, typename S, typename C>
__device__ __forceinline__ void ens_dataflow(const EnsPlan& p, long long gw) {
  const int lane = threadIdx.x & 31;
  const int R = p.remap_every;
  const int P = p.nsteps * 10 + (R > 0 ? (p.nsteps / R) * 3 : 0);
  int start = (int)(gw % p.nm);
  long long idle0 = global_ns();
  while (true) {
    int m = -1, ph = 0;
    long long item = 0;
    if (lane == 0) {
      for (int t = 0; t < p.nm; ++t) {
        int mm = start + t;
        if (mm >= p.nm) mm -= p.nm;
        const unsigned long long tk = *(volatile unsigned long long*)(p.tk + mm);
        const int ph0 = (int)(tk >> 32);
        if (ph0 >= P) continue;
        int st0, fl0;
        ens_phase(ph0, R, st0, fl0);
        if ((long long)(tk & 0xffffffffull) >= ens_count(p, st0, mm)) continue;
        const unsigned long long old = atomicAdd(p.tk + mm, 1ull);
        const int ph1 = (int)(old >> 32);
        if (ph1 >= P) continue;
        int st1, fl1;
        ens_phase(ph1, R, st1, fl1);
        const long long it1 = (long long)(old & 0xffffffffull);
        if (it1 >= ens_count(p, st1, mm)) continue;
        m = mm;
        ph = ph1;
        item = it1;
        break;
      }
    }
    m = __shfl_sync(0xffffffffu, m, 0);
    if (m < 0) {
      int stop = 0;
      if (lane == 0) {
        if (*(volatile unsigned*)p.fin >= (unsigned)p.nm || *(volatile int*)p.err != 0) {
          stop = 1;
        } else if (global_ns() - idle0 > p.timeout_ns) {
          atomicOr(p.err, 1);
          stop = 1;
        } else {
          __nanosleep(256);
        }
      }
      if (__shfl_sync(0xffffffffu, stop, 0)) return;
      continue;
    }
    ph = __shfl_sync(0xffffffffu, ph, 0);
    item = __shfl_sync(0xffffffffu, item, 0);
    idle0 = global_ns();
    start = m;
    __threadfence();  // acquire: the member's earlier phases
    int stage, flip;
    ens_phase(ph, R, stage, flip);
    const EnsMember& M = p.m[m];
    ens_item<T, S, C>(stage, M, M.cur0 ^ flip, item);
    __threadfence();  // release: this item's writes
    __syncwarp();
    if (lane == 0) {
      const unsigned done = atomicAdd(p.dn + m, 1u) + 1u;
      if ((long long)done == ens_count(p, stage, m)) {
        atomicExch(p.dn + m, 0u);
        __threadfence();
        if (ph + 1 >= P) atomicAdd(p.fin, 1u);
        atomicExch(p.tk + m, (unsigned long long)(ph + 1) << 32);
      }
    }
    __syncwarp();
  }
}

// The run: p.nsteps steps of every member, the remap on steps whose number
// (counted from 1 at the launch) is a multiple of p.remap_every.
template <typename T, typename S, typename C>
__global__ void __launch_bounds__(MW * MWARPS, 3) k_ensemble(EnsPlan p) {
  const long long nwarps = (long long)gridDim.x * MWARPS;
  const long long gw = (long long)blockIdx.x * MWARPS + (threadIdx.x >> 5);
  if (p.dataflow) {
    if (p.nm > 0) ens_dataflow<T, S, C>(p, gw);
    return;
  }
  int flip = 0;  // swaps of the time levels so far (the same for every member)
  const bool timer = p.stage_ns != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
  long long tprev = timer ? global_ns() : 0;
  for (int s = 0; s < p.nsteps; ++s) {
    const bool remap = p.remap_every > 0 && (s + 1) % p.remap_every == 0;
    for (int stage = 0; stage < E_NSTAGE; ++stage) {
      if (!remap && (stage == E_RRING || stage == E_RWIND || stage == E_RENER)) continue;
      const long long* off = p.off + (long long)stage * (p.nm + 1);
      const long long total = off[p.nm];
      for (long long it = gw; it < total; it += nwarps) {
        const int m = ens_member(off, p.nm, it);
        const EnsMember& M = p.m[m];
        ens_item<T, S, C>(stage, M, M.cur0 ^ flip, it - off[m]);
      }
      if (stage == E_DMOM || stage == E_RENER) flip ^= 1;
      if (!ens_barrier(p)) return;
      if (timer) {
        const long long t = global_ns();
        atomicAdd(p.stage_ns + stage, (unsigned long long)(t - tprev));
        tprev = t;
      }
    }
  }
}

}  // namespace atm
