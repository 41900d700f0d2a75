// sweep3d.cuh -- one launch per time step for the 3D Yee solver: E and H
// updated in a single sweep over x-planes, each plane of a CTA's tile staged
// in shared memory by TMA (cp.async.bulk.tensor, no multicast).
//
// Work item = (y0, z0, x0, x1) of one job.  The CTA has TBY x TBZ threads; thread
// (ey, ez) is cell y = y0 - 1 + ey, z = z0 - 1 + ez for every plane of the
// item.  Cells with ey, ez >= 1 are owned (the tile is (TBY-1) x (TBZ-1)); row
// ey = 0 and column ez = 0 are the low halo, whose new E the tile recomputes
// because its H update needs E(j-1) and E(k-1) -- so tiles never exchange
// data within a step.  Per plane i the CTA needs H(i) and H(i+1) over the
// box rows y0-1 .. y0+TBY-1 and columns z0-1 .. z0+TBZ-1, plus E(i) and dt/eps(i);
// it writes new E and H of its owned cells to the other buffer (ping-pong).
// Every field word is read once and written once per step from HBM (60 B per
// cell in FP32); halo re-reads hit L2.
//
// A thread keeps its cell's old H and new E in registers from the E half to
// the H half, and its new Ey, Ez for the next plane (the x-differences of the
// H update); in-plane E neighbours come from a double-buffered shared tile.
// Range tests, CPML slab positions and kappa*dx factors that depend on (j, k)
// are computed once per work item, those that depend on i once per plane.
// Operand order equals kernels.cuh (y3_e_compute / y3_h_compute), which
// follows the reference kernels, so OIDT_ARITH_EXACT results match bit for bit.
//
// TMA boxes start at z = floor4(z0 - 1) (16-byte aligned x-coordinate) and
// y = y0 - 1; out-of-range rows/columns read as zero.  Waits on the TMA
// mbarriers are bounded (kWaitCycles): on expiry the CTA records an error in
// state[1], stops issuing, waits the same bound for copies in flight, returns.
#pragma once
#include <cuda.h>

#include "kernels.cuh"

namespace oidt {

struct SweepItem {
  int y0, z0, x0, x1;
};

// E-box of the CTA: TBY x TBZ threads, owned tile (TBY-1) x (TBZ-1).
constexpr int kSweepEY = 8, kSweepEZ = 32, kSweepStages = 3;
constexpr int kSweepTY = kSweepEY - 1, kSweepTZ = kSweepEZ - 1;  // owned tile
constexpr long long kWaitCycles = 4000000000LL;                  // ~2 s at 1.9 GHz

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

template <typename T, int TBY, int TBZ> struct SweepGeom {
  static constexpr int BY = TBY + 1;         // box rows: y0-1 .. y0+TBY-1
  static constexpr int BZ = TBZ + 8;         // box cols from floor4(z0-1): covers z0-1 .. z0+TBZ-1 (+3 slack)
  static constexpr int BOX = BY * BZ;
  static constexpr int BOXS = (int)(((BOX * sizeof(T) + 127) / 128) * 128 / sizeof(T));  // 128-B aligned boxes
  static constexpr int NT = TBY * TBZ;
};

template <typename T, int TBY, int TBZ, int S>
constexpr size_t sweep_smem_bytes() {
  using G = SweepGeom<T, TBY, TBZ>;
  return (size_t)S * 9 * G::BOXS * sizeof(T) + 2 * 3 * G::NT * sizeof(T) + 8 * S + 2 * 128;
}

// Packed CPML slab position: q (coefficient index) | d << 12 | side << 24, or -1.
__device__ __forceinline__ int slab_code_e(int c, int b, int e, int P) {
  int d, side;
  const int q = e_slab(c, b, e, P, d, side);
  return q < 0 ? -1 : (q | (d << 12) | (side << 24));
}
__device__ __forceinline__ int slab_code_h(int c, int b, int e, int P) {
  int d, side;
  const int q = h_slab(c, b, e, P, d, side);
  return q < 0 ? -1 : (q | (d << 12) | (side << 24));
}
__device__ __forceinline__ int sq(int code) { return code & 0xfff; }
__device__ __forceinline__ int sd(int code) { return (code >> 12) & 0xfff; }
__device__ __forceinline__ int ss(int code) { return code >> 24; }

// `p` is the job's view for this step (which buffer is old and which is
// new), passed in the kernel's parameter space so every field is a constant
// operand; `items` is the job's tile table.
template <typename T, bool EXACT, int TBY, int TBZ, int S>
__global__ void __launch_bounds__(TBY *TBZ) k_sweep3d(const __grid_constant__ Params<T> p,
                                                    const SweepItem *__restrict__ items, int s) {
  using G = SweepGeom<T, TBY, TBZ>;
  using A = Ar<T, EXACT>;
  constexpr int NT = G::NT, BZ = G::BZ, BOX = G::BOX, BOXS = G::BOXS;
  constexpr unsigned STAGE_BYTES = 9u * BOX * sizeof(T);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  T *stage = reinterpret_cast<T *>(smem);
  T *sE = stage + S * 9 * BOXS;  // [2][3][NT]
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(
      (reinterpret_cast<uintptr_t>(sE + 2 * 3 * NT) + 127) & ~uintptr_t(127));
  __shared__ int s_abort, s_issued, s_failed;

  const SweepItem it = items[blockIdx.x];
  const int tid = threadIdx.x;
  const int ey = tid / TBZ, ez = tid % TBZ;
  const int y0 = it.y0, z0 = it.z0, x0 = it.x0, x1 = it.x1;
  const int zb = (z0 - 1) & ~3;  // box column origin (floor to a multiple of 4)
  const int zoff = (z0 - 1) - zb;
  const int xs = x0 - 1;            // first plane loaded (E of x0-1 feeds H of x0)
  const int nplanes = x1 - xs + 1;  // planes xs .. x1
  const int n = p.state[0] + s;
  const int y = y0 - 1 + ey, z = z0 - 1 + ez;
  const bool ingrid = y >= 0 && y < p.ny && z >= 0 && z < p.nz;
  const bool own = ingrid && ey >= 1 && ez >= 1;
  const int bo = ey * BZ + ez + zoff;  // this cell in a box
  const int P = p.P;

  // ---- per-item (j, k) classification --------------------------------------
  const bool jin_c = y >= p.jb && y < p.je, jin_o = y > p.jb && y < p.je;   // [jb,je) and (jb,je)
  const bool kin_c = z >= p.kb && z < p.ke, kin_o = z > p.kb && z < p.ke;
  const bool ex_jk = ingrid && jin_c && kin_c;   // Ex: j [jb,je), k [kb,ke)
  const bool ey_jk = ingrid && jin_o && kin_c;   // Ey: j (jb,je), k [kb,ke)
  const bool ez_jk = ingrid && jin_c && kin_o;   // Ez: j [jb,je), k (kb,ke)
  const bool hx_jk = own && jin_o && kin_o;      // Hx: j (jb,je), k (kb,ke)
  const bool hy_jk = own && jin_c && kin_o;      // Hy: j [jb,je), k (kb,ke)
  const bool hz_jk = own && jin_o && kin_c;      // Hz: j (jb,je), k [kb,ke)
  const int ye_code = ingrid ? slab_code_e(y, p.jb, p.je, P) : -1;
  const int ze_code = ingrid ? slab_code_e(z, p.kb, p.ke, P) : -1;
  const int yh_code = own ? slab_code_h(y, p.jb, p.je, P) : -1;
  const int zh_code = own ? slab_code_h(z, p.kb, p.ke, P) : -1;
  const int yc = ingrid ? y : 0, zc = ingrid ? z : 0;
  const T kye = EXACT ? p.kd[1][yc] : T(0), rkye = p.rkd[1][yc];
  const T kze = EXACT ? p.kd[2][zc] : T(0), rkze = p.rkd[2][zc];
  const T kyh = EXACT ? p.kd[4][yc] : T(0), rkyh = p.rkd[4][yc];
  const T kzh = EXACT ? p.kd[5][zc] : T(0), rkzh = p.rkd[5][zc];
  const bool src_jk = p.src_field >= 0 && y >= p.slo[1] && y < p.shi[1] && z >= p.slo[2] && z < p.shi[2];
  const bool src_jk1 = p.src_field == HY && y >= p.slo[1] && y < p.shi[1] && z + 1 >= p.slo[2] && z + 1 < p.shi[2];
  const bool capt = own && (z == p.port_pos[0] || z == p.port_pos[1] || z == p.port_pos[0] + 1 ||
                            z == p.port_pos[1] + 1);
  const long long g_jk = (long long)y * p.nzp + z;  // cell offset inside a plane

  const unsigned char *tmf = static_cast<const unsigned char *>(p.tmap_f);
  const unsigned char *tmc = static_cast<const unsigned char *>(p.tmap_cb);
  auto issue = [&](int u) {  // load plane xs+u into stage u % S
    T *dst = stage + (u % S) * 9 * BOXS;
    unsigned long long *b = bar + (u % S);
    fence_proxy_async();
    mbar_expect_tx(b, STAGE_BYTES);
    const int xi = xs + u;
    for (int f = 0; f < 6; ++f) tma_load_3d(dst + f * BOXS, tmf + f * 128, zb, y0 - 1, xi, b);
    for (int a = 0; a < 3; ++a) tma_load_3d(dst + (6 + a) * BOXS, tmc + a * 128, zb, y0 - 1, xi, b);
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

  if (tid == 0) {
    s_abort = 0;
    s_failed = 0x7fffffff;
    for (int k = 0; k < S; ++k) mbar_init(bar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    int u = 0;
    for (; u < S - 1 && u < nplanes; ++u) issue(u);
    s_issued = u;
  }
  bool ok = wait(0);
  if (!ok) atomicMin(&s_failed, 0);
  T ey_prev = T(0), ez_prev = T(0);  // new Ey, Ez of this cell at the previous plane

  for (int u = 0; u + 1 < nplanes; ++u) {
    const int i = xs + u;
    if (ok && !(ok = wait(u + 1))) atomicMin(&s_failed, u + 1);
    const T *cur = stage + (u % S) * 9 * BOXS;
    const T *nxt = stage + ((u + 1) % S) * 9 * BOXS;
    T *enew = sE + (u & 1) * 3 * NT;
    // ---- per-plane values ----------------------------------------------------
    const bool i_c = i >= p.ib && i < p.ie, i_o = i > p.ib && i < p.ie;
    const int xe_code = slab_code_e(i, p.ib, p.ie, P);
    const int xh_code = slab_code_h(i, p.ib, p.ie, P);
    const T kxe = EXACT ? p.kd[0][i] : T(0), rkxe = p.rkd[0][i];
    const T kxh = EXACT ? p.kd[3][i] : T(0), rkxh = p.rkd[3][i];
    const bool src_i = i >= p.slo[0] && i < p.shi[0];
    const bool src_i1 = i + 1 >= p.slo[0] && i + 1 < p.shi[0];
    const T Jn = p.src_field >= 0 ? p.jsrc[n] : T(0);
    // ---- new E of this cell (all threads of the E box) ------------------------
    T hx0 = T(0), hy0 = T(0), hz0 = T(0), e0 = T(0), e1 = T(0), e2 = T(0);
    int me = 0;
    if (ok && ingrid) {
      hx0 = cur[HX * BOXS + bo];
      hy0 = cur[HY * BOXS + bo];
      hz0 = cur[HZ * BOXS + bo];
      e0 = cur[EX * BOXS + bo];
      e1 = cur[EY * BOXS + bo];
      e2 = cur[EZ * BOXS + bo];
      const bool wpsi = own && i >= x0;  // this CTA owns the cell's new psi
      if (i_o && ex_jk) {  // Ex                                     fdtd_funcs.py:43-50, 113-136
        const T cb = cur[(6 + 0) * BOXS + bo];
        const T dhz = A::sub(cur[HZ * BOXS + bo + BZ], hz0);
        const T hy1 = cur[HY * BOXS + bo + 1];
        const T dhy = A::sub(hy1, hy0);
        T e = A::add(e0, A::mul(cb, A::sub(A::div(dhz, kye, rkye), A::div(dhy, kze, rkze))));
        if (ye_code >= 0) {
          const int q = sq(ye_code);
          const long long o = psi_idx3(AY, i, sd(ye_code), z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.be[q], p.psi[EX][AY][ss(ye_code)][o]), A::div(A::mul(p.ce[q], dhz), p.dx, p.rdx));
          if (wpsi) p.psin[EX][AY][ss(ye_code)][o] = v;
          e = A::add(e, A::mul(cb, v));
        }
        if (ze_code >= 0) {
          T h1 = hy1, h0 = hy0;
          if (p.src_field == HY) {
            if (src_i && src_jk1) h1 = A::sub(h1, Jn);
            if (src_i && src_jk) h0 = A::sub(h0, Jn);
          }
          const int q = sq(ze_code);
          const long long o = psi_idx3(AZ, i, y, sd(ze_code), p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.be[q], p.psi[EX][AZ][ss(ze_code)][o]),
                             A::div(A::mul(p.ce[q], A::sub(h1, h0)), p.dx, p.rdx));
          if (wpsi) p.psin[EX][AZ][ss(ze_code)][o] = v;
          e = A::sub(e, A::mul(cb, v));
        }
        e0 = e;
        me |= 1;
      }
      if (i_c && ey_jk) {  // Ey                                     :53-60, 104-110, 139-162
        const T cb = cur[(6 + 1) * BOXS + bo];
        const T dhx = A::sub(cur[HX * BOXS + bo + 1], hx0);
        const T dhz = A::sub(nxt[HZ * BOXS + bo], hz0);
        T e = A::add(e1, A::mul(cb, A::sub(A::div(dhx, kze, rkze), A::div(dhz, kxe, rkxe))));
        if (p.src_field == EY && src_i && src_jk) e = A::sub(e, Jn);
        if (xe_code >= 0) {
          const int q = sq(xe_code);
          const long long o = psi_idx3(AX, sd(xe_code), y, z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.be[q], p.psi[EY][AX][ss(xe_code)][o]), A::div(A::mul(p.ce[q], dhz), p.dx, p.rdx));
          if (wpsi) p.psin[EY][AX][ss(xe_code)][o] = v;
          e = A::sub(e, A::mul(cb, v));
        }
        if (ze_code >= 0) {
          const int q = sq(ze_code);
          const long long o = psi_idx3(AZ, i, y, sd(ze_code), p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.be[q], p.psi[EY][AZ][ss(ze_code)][o]), A::div(A::mul(p.ce[q], dhx), p.dx, p.rdx));
          if (wpsi) p.psin[EY][AZ][ss(ze_code)][o] = v;
          e = A::add(e, A::mul(cb, v));
        }
        e1 = e;
        me |= 2;
      }
      if (i_c && ez_jk) {  // Ez                                     :63-70, 165-188
        const T cb = cur[(6 + 2) * BOXS + bo];
        const T hy1 = nxt[HY * BOXS + bo];
        const T dhy = A::sub(hy1, hy0);
        const T dhx = A::sub(cur[HX * BOXS + bo + BZ], hx0);
        T e = A::add(e2, A::mul(cb, A::sub(A::div(dhy, kxe, rkxe), A::div(dhx, kye, rkye))));
        if (xe_code >= 0) {
          T h1 = hy1, h0 = hy0;
          if (p.src_field == HY) {
            if (src_i1 && src_jk) h1 = A::sub(h1, Jn);
            if (src_i && src_jk) h0 = A::sub(h0, Jn);
          }
          const int q = sq(xe_code);
          const long long o = psi_idx3(AX, sd(xe_code), y, z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.be[q], p.psi[EZ][AX][ss(xe_code)][o]),
                             A::div(A::mul(p.ce[q], A::sub(h1, h0)), p.dx, p.rdx));
          if (wpsi) p.psin[EZ][AX][ss(xe_code)][o] = v;
          e = A::add(e, A::mul(cb, v));
        }
        if (ye_code >= 0) {
          const int q = sq(ye_code);
          const long long o = psi_idx3(AY, i, sd(ye_code), z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.be[q], p.psi[EZ][AY][ss(ye_code)][o]), A::div(A::mul(p.ce[q], dhx), p.dx, p.rdx));
          if (wpsi) p.psin[EZ][AY][ss(ye_code)][o] = v;
          e = A::sub(e, A::mul(cb, v));
        }
        e2 = e;
        me |= 4;
      }
    }
    enew[tid] = e0;
    enew[NT + tid] = e1;
    enew[2 * NT + tid] = e2;
    if (!ok) s_abort = 1;
    __syncthreads();  // new E of the tile visible; stage (u-1) % S no longer read
    if (s_abort) break;
    if (tid == 0 && u + S - 1 < nplanes) {
      issue(u + S - 1);  // into stage (u-1) % S
      s_issued = u + S;
    }
    // ---- new H of owned cells; store E and H ------------------------------------
    if (own && i >= x0) {
      T h0v = hx0, h1v = hy0, h2v = hz0;
      int mh = 0;
      const T db = p.db;
      if (i_c && hx_jk) {  // Hx                                     :73-80, 191-214
        const T dey = A::sub(e1, enew[NT + tid - 1]);
        const T dez = A::sub(e2, enew[2 * NT + tid - TBZ]);
        T h = A::add(h0v, A::mul(db, A::sub(A::div(dey, kzh, rkzh), A::div(dez, kyh, rkyh))));
        if (yh_code >= 0) {
          const int q = sq(yh_code);
          T *ps = p.psi[HX][AY][ss(yh_code)] + psi_idx3(AY, i, sd(yh_code), z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dez), p.dx, p.rdx));
          *ps = v;
          h = A::sub(h, A::mul(db, v));
        }
        if (zh_code >= 0) {
          const int q = sq(zh_code);
          T *ps = p.psi[HX][AZ][ss(zh_code)] + psi_idx3(AZ, i, y, sd(zh_code), p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dey), p.dx, p.rdx));
          *ps = v;
          h = A::add(h, A::mul(db, v));
        }
        h0v = h;
        mh |= 1;
      }
      if (i_o && hy_jk) {  // Hy                                     :83-90, 217-240
        const T dez = A::sub(e2, ez_prev);
        const T dex = A::sub(e0, enew[tid - 1]);
        T h = h1v;
        if (p.src_field == HY && src_i && src_jk) h = A::sub(h, Jn);  // source precedes update_hy
        h = A::add(h, A::mul(db, A::sub(A::div(dez, kxh, rkxh), A::div(dex, kzh, rkzh))));
        if (xh_code >= 0) {
          const int q = sq(xh_code);
          T *ps = p.psi[HY][AX][ss(xh_code)] + psi_idx3(AX, sd(xh_code), y, z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dez), p.dx, p.rdx));
          *ps = v;
          h = A::add(h, A::mul(db, v));
        }
        if (zh_code >= 0) {
          const int q = sq(zh_code);
          T *ps = p.psi[HY][AZ][ss(zh_code)] + psi_idx3(AZ, i, y, sd(zh_code), p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dex), p.dx, p.rdx));
          *ps = v;
          h = A::sub(h, A::mul(db, v));
        }
        h1v = h;
        mh |= 2;
      }
      if (i_o && hz_jk) {  // Hz                                     :93-100, 243-266
        const T dex = A::sub(e0, enew[tid - TBZ]);
        const T dey = A::sub(e1, ey_prev);
        T h = A::add(h2v, A::mul(db, A::sub(A::div(dex, kyh, rkyh), A::div(dey, kxh, rkxh))));
        if (xh_code >= 0) {
          const int q = sq(xh_code);
          T *ps = p.psi[HZ][AX][ss(xh_code)] + psi_idx3(AX, sd(xh_code), y, z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dey), p.dx, p.rdx));
          *ps = v;
          h = A::sub(h, A::mul(db, v));
        }
        if (yh_code >= 0) {
          const int q = sq(yh_code);
          T *ps = p.psi[HZ][AY][ss(yh_code)] + psi_idx3(AY, i, sd(yh_code), z, p.nx, p.ny, p.nz, P);
          const T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dex), p.dx, p.rdx));
          *ps = v;
          h = A::add(h, A::mul(db, v));
        }
        h2v = h;
        mh |= 4;
      }
      const long long g = (long long)i * p.ny * p.nzp + g_jk;
      p.fn[EX][g] = e0;
      p.fn[EY][g] = e1;
      p.fn[EZ][g] = e2;
      p.fn[HX][g] = h0v;
      p.fn[HY][g] = h1v;
      p.fn[HZ][g] = h2v;
      if (capt) {
        const T ev[3] = {e0, e1, e2}, hv[3] = {h0v, h1v, h2v};
        y3_capture_e(p, s, i, y, z, me, ev);
        y3_capture_h(p, s, i, y, z, mh, hv);
      }
    }
    ey_prev = e1;
    ez_prev = e2;
  }
  if (s_abort && tid == 0) {
    atomicExch(p.state + 1, 1);  // reported to the host by oidt_job_sync
    // copies issued after the failed one: bounded wait so none lands after exit
    for (int u = s_failed; u < s_issued; ++u) (void)wait(u);
  }
}

}  // namespace oidt
