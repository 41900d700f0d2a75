// sweep3d.cuh -- one launch per time step for the 3D Yee solver: E and H
// updated in a single sweep over x-planes, each plane of a CTA's tile staged
// in shared memory by TMA (cp.async.bulk.tensor, no multicast).
//
// Work item = (job, y0, z0, x0, x1): the CTA owns cells y in [y0, y0+TY),
// z in [z0, z0+TZ) of planes x in [x0, x1).  Per plane i it needs, from the
// old buffers, H(i) and H(i+1) over a one-cell halo and E(i), dt/eps(i) over
// the low halo; it computes the new E over the tile plus its low halo (the
// halo cells recompute what the neighbouring tile computes, so no exchange
// is needed), then the new H of its own cells, and writes new E and H to the
// other buffer (ping-pong).  Every field word is read once and written once
// per step from HBM (60 B per cell in FP32); halo re-reads hit L2.
//
// Shared memory per CTA: S stages x 9 boxes [TY+2][TZ+8] (fields + dt/eps of
// one plane; z starts 4 cells before z0 so the TMA x-coordinate stays 16-byte
// aligned) + two planes of new E over the tile + low halo.
//
// Waits on the TMA mbarriers are bounded: after kWaitCycles clock cycles the
// CTA records an error in state[1], stops issuing work, gives the copies still
// in flight the same bounded time to land, and returns.
#pragma once
#include <cuda.h>

#include "kernels.cuh"

namespace oidt {

struct SweepItem {
  int job, y0, z0, x0, x1;
};

constexpr int kSweepTY = 8, kSweepTZ = 32, kSweepStages = 3;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz: bounded TMA wait

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int c0, int c1, int c2,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory accessor for one cell of the tile.
template <typename T, int TY, int TZ> struct BoxAcc3 {
  static constexpr int BY = TY + 2, BZ = TZ + 8, BOX = BY * BZ, EY_ = TY + 1, EZ_ = TZ + 1, EBOX = EY_ * EZ_;
  // box stride in shared memory: each TMA destination starts 128-byte aligned
  static constexpr int BOXS = (int)(((BOX * sizeof(T) + 127) / 128) * 128 / sizeof(T));
  const T *cur;   // stage of plane i: 9 boxes
  const T *nxt;   // stage of plane i+1
  const T *enew;  // new E of plane i: 3 x [EY_][EZ_]
  const T *eprv;  // new E of plane i-1
  int bo;         // box offset of the cell: (y-(y0-1))*BZ + (z-(z0-4))
  int eo;         // E-box offset of the cell: (y-(y0-1))*EZ_ + (z-(z0-1))
  __device__ __forceinline__ T h(int f, int di, int dj, int dk) const {
    return (di ? nxt : cur)[f * BOXS + bo + dj * BZ + dk];
  }
  __device__ __forceinline__ T e(int f, int di, int dj, int dk) const {
    return di ? eprv[f * EBOX + eo] : enew[f * EBOX + eo + dj * EZ_ + dk];
  }
  __device__ __forceinline__ T eold(int f) const { return cur[f * BOXS + bo]; }
  __device__ __forceinline__ T hold(int f) const { return cur[f * BOXS + bo]; }
  __device__ __forceinline__ T cb(int a) const { return cur[(6 + a) * BOXS + bo]; }
};

template <typename T, int TY, int TZ, int S>
constexpr size_t sweep_smem_bytes() {
  return (size_t)S * 9 * BoxAcc3<T, TY, TZ>::BOXS * sizeof(T) + 2 * 3 * (TY + 1) * (TZ + 1) * sizeof(T) +
         sizeof(Params<T>) + 8 * S + 3 * 128;
}

// params[job] holds the parity-0 and parity-1 views of each job (which
// buffer is old and which is new); `par` selects one for this step.
template <typename T, bool EXACT, int TY, int TZ, int S>
__global__ void __launch_bounds__(TY *TZ) k_sweep3d(const Params<T> *__restrict__ params, const int *__restrict__ par0,
                                                    const SweepItem *__restrict__ items, int par, int s) {
  using Acc = BoxAcc3<T, TY, TZ>;
  constexpr int NT = TY * TZ, BOX = Acc::BOX, BOXS = Acc::BOXS, BZ = Acc::BZ, EZ_ = Acc::EZ_, EBOX = Acc::EBOX;
  constexpr unsigned STAGE_BYTES = 9u * BOX * sizeof(T);
  static_assert(sizeof(Params<T>) % 8 == 0, "Params must be a whole number of 8-byte words");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  T *stage = reinterpret_cast<T *>(smem);
  T *sE = stage + S * 9 * BOXS;
  unsigned long long *sp = reinterpret_cast<unsigned long long *>(
      (reinterpret_cast<uintptr_t>(sE + 2 * 3 * EBOX) + 127) & ~uintptr_t(127));
  unsigned long long *bar = sp + sizeof(Params<T>) / 8;
  __shared__ int s_abort;

  const SweepItem it = items[blockIdx.x];
  const int tid = threadIdx.x;
  {
    const unsigned long long *src =
        reinterpret_cast<const unsigned long long *>(params + 2 * it.job + ((par ^ par0[it.job]) & 1));
    for (int w = tid; w < (int)(sizeof(Params<T>) / 8); w += NT) sp[w] = src[w];
  }
  __syncthreads();  // the parameter copy must be complete before any thread reads it
  const Params<T> &p = *reinterpret_cast<const Params<T> *>(sp);
  const int y0 = it.y0, z0 = it.z0, x0 = it.x0, x1 = it.x1;
  const int xs = x0 - 1;          // first plane loaded (E of x0-1 feeds H of x0)
  const int nplanes = x1 - xs + 1;  // planes xs .. x1
  const int n = p.state[0] + s;
  const unsigned char *tmf = static_cast<const unsigned char *>(p.tmap_f);
  const unsigned char *tmc = static_cast<const unsigned char *>(p.tmap_cb);

  auto issue = [&](int u) {  // load plane xs+u into stage u % S
    T *dst = stage + (u % S) * 9 * BOXS;
    unsigned long long *b = bar + (u % S);
    fence_proxy_async();
    mbar_expect_tx(b, STAGE_BYTES);
    const int xi = xs + u;
    for (int f = 0; f < 6; ++f) tma_load_3d(dst + f * BOXS, tmf + f * 128, z0 - 4, y0 - 1, xi, b);
    for (int a = 0; a < 3; ++a) tma_load_3d(dst + (6 + a) * BOXS, tmc + a * 128, z0 - 4, y0 - 1, xi, b);
  };
  auto wait = [&](int u) -> bool {
    unsigned long long *b = bar + (u % S);
    const unsigned ph = (unsigned)((u / S) & 1);
    const long long t0 = clock64();
    while (!mbar_try_wait(b, ph)) {
      if (clock64() - t0 > kWaitCycles) return false;
    }
    return true;
  };
  __shared__ int s_issued, s_failed;

  if (tid == 0) {
    s_abort = 0;
    for (int k = 0; k < S; ++k) mbar_init(bar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    s_issued = 0;
    s_failed = 0x7fffffff;
    for (int u = 0; u < S && u < nplanes; ++u) issue(u), s_issued = u + 1;
  }
  __syncthreads();

  bool ok = wait(0);
  if (!ok) atomicMin(&s_failed, 0);
  for (int u = 0; u + 1 < nplanes; ++u) {  // plane i = xs + u, needs stage u and u+1
    const int i = xs + u;
    if (ok && !(ok = wait(u + 1))) atomicMin(&s_failed, u + 1);
    if (!ok) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    const T *cur = stage + (u % S) * 9 * BOXS;
    const T *nxt = stage + ((u + 1) % S) * 9 * BOXS;
    T *enew = sE + (u & 1) * 3 * EBOX;
    const T *eprv = sE + ((u + 1) & 1) * 3 * EBOX;
    // ---- new E over the tile and its low halo -----------------------------
    for (int e = tid; e < EBOX; e += NT) {
      const int ey = e / EZ_, ez = e % EZ_;
      const int y = y0 - 1 + ey, z = z0 - 1 + ez;
      T ev[3] = {T(0), T(0), T(0)};
      if (y >= 0 && y < p.ny && z >= 0 && z < p.nz) {
        Acc a{cur, nxt, enew, eprv, ey * BZ + ez + 3, e};
        const bool own = ey >= 1 && ez >= 1 && i >= x0;
        y3_e_compute<T, EXACT>(p, a, i, y, z, n, own, ev);
      }
      enew[e] = ev[0];
      enew[EBOX + e] = ev[1];
      enew[2 * EBOX + e] = ev[2];
    }
    __syncthreads();
    // ---- new H of the tile's cells; store E and H ---------------------------
    if (i >= x0) {
      for (int c = tid; c < TY * TZ; c += NT) {
        const int ty = c / TZ, tz = c % TZ;
        const int y = y0 + ty, z = z0 + tz;
        if (y >= p.ny || z >= p.nz) continue;
        const int eo = (ty + 1) * EZ_ + tz + 1;
        Acc a{cur, nxt, enew, eprv, (ty + 1) * BZ + tz + 4, eo};
        T hv[3];
        const int mh = y3_h_compute<T, EXACT>(p, a, i, y, z, n, hv);
        const long long g = ((long long)i * p.ny + y) * p.nzp + z;
        const T ev[3] = {enew[eo], enew[EBOX + eo], enew[2 * EBOX + eo]};
        p.fn[EX][g] = ev[0];
        p.fn[EY][g] = ev[1];
        p.fn[EZ][g] = ev[2];
        p.fn[HX][g] = hv[0];
        p.fn[HY][g] = hv[1];
        p.fn[HZ][g] = hv[2];
        if (z == p.port_pos[0] || z == p.port_pos[1] || z == p.port_pos[0] + 1 || z == p.port_pos[1] + 1) {
          // capture only components the step updated (the others stay zero)
          const int me = (i > p.ib && i < p.ie && y >= p.jb && y < p.je && z >= p.kb && z < p.ke ? 1 : 0) |
                         (i >= p.ib && i < p.ie && y > p.jb && y < p.je && z >= p.kb && z < p.ke ? 2 : 0);
          y3_capture_e(p, s, i, y, z, me, ev);
          y3_capture_h(p, s, i, y, z, mh, hv);
        }
      }
    }
    __syncthreads();
    if (tid == 0 && u + S < nplanes) issue(u + S), s_issued = u + S + 1;  // stage u is free now
  }
  if (s_abort && tid == 0) {
    atomicExch(p.state + 1, 1);  // reported to the host by oidt_job_sync
    // copies issued after the failed one: bounded wait so none lands after exit
    for (int u = s_failed; u < s_issued; ++u) (void)wait(u);
  }
}

}  // namespace oidt
