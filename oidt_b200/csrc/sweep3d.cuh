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
// mbarriers are bounded (p.wait_cycles, kWaitCycles unless a test lowers it):
// on expiry the CTA records an error in state[1], stops issuing, waits for the
// copies it has in flight (each wait bounded by kWaitCycles: every copy is a
// valid load that lands) and returns, so nothing is written into its shared
// memory after it exits.
#pragma once
#include <cuda.h>

#include <type_traits>

#include "kernels.cuh"

namespace oidt {

// Work item flags, CTA-uniform, set on the host per item.  Every plane runs
// the three curl updates of each component unconditionally; the source, the
// CPML terms, the DFT capture and the per-cell range masks are each behind a
// branch on these flags (or on the plane index), so a plane of an unflagged
// item outside both x CPML slabs runs no per-cell test at all.
enum : int {
  kItemEdge = 1,   // some E-box cell lies outside (jb, je) x (kb, ke) (or outside the grid)
  kItemYSlab = 2,  // some E-box cell lies in a y CPML slab
  kItemZSlab = 4,  // some E-box cell lies in a z CPML slab
  kItemSrc = 8,    // the source box meets the item's (y, z) columns
  kItemPort = 16,  // an owned column lies on a port plane (DFT capture)
};

struct SweepItem {
  int y0, z0, x0, x1;
  int flags, pad0, pad1, pad2;
};

// E-box of the CTA: TBY x TBZ threads, owned tile (TBY-1) x (TBZ-1).
constexpr int kSweepEY = 8, kSweepEZ = 32, kSweepStages = 3;
constexpr int kSweepTY = kSweepEY - 1, kSweepTZ = kSweepEZ - 1;  // owned tile

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
// Non-blocking probe (mbarrier.try_wait may suspend the thread until the
// phase completes; a short bound needs probes that return at once).
__device__ __forceinline__ bool mbar_test_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
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
  static constexpr int NT = TBY * TBZ;                      // cells of the E box
  static constexpr int THREADS = NT;                        // one thread per cell
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
// new), passed in the kernel's parameter space; `items` is the job's tile
// table.
//
// Pipeline: S stages of plane boxes.  Plane u+1 must be resident when plane u
// is processed (the E update reads H(i+1)); the stage of plane u is refilled
// with plane u+S right after the barrier that ends plane u's E half, so loads
// run S-1 planes ahead.
//
// Items without flags (every E-box cell strictly inside the update ranges
// and outside the y and z CPML slabs, no source, no port) run a specialised
// march whose only decisions are per plane (boundary planes, x CPML planes);
// flagged items run the general march with per-cell range masks.
template <typename T, bool EXACT, int TBY, int TBZ, int S>
__global__ void __launch_bounds__(TBY *TBZ, sizeof(T) == 4 ? 4 : 2)
    k_sweep3d(const __grid_constant__ Params<T> p, const SweepItem *__restrict__ items, int s) {
  pdl_wait();
  static_assert(S >= 3, "the stage refilled after plane u must differ from those of planes u+1, u+2");
  using G = SweepGeom<T, TBY, TBZ>;
  using A = Ar<T, EXACT>;
  constexpr int NT = G::NT, BZ = G::BZ, BOX = G::BOX, BOXS = G::BOXS, SB = 9 * BOXS;
  constexpr unsigned STAGE_BYTES = 9u * BOX * sizeof(T);
  // Shared memory is addressed as offsets from the __shared__ array itself
  // (no integer round trip), so every access compiles to a shared load/store.
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const unsigned pad = (128u - (smem_u32(smem_raw) & 127u)) & 127u;
  T *const stage = reinterpret_cast<T *>(smem_raw + pad);  // [S][9][BOXS]
  T *const sE = stage + S * SB;                              // [2][3][NT]
  unsigned long long *const bar = reinterpret_cast<unsigned long long *>(sE + 2 * 3 * NT);
  __shared__ int s_abort[2], s_issued, s_failed;  // s_abort[u & 1]: plane u's verdict

  const SweepItem it = items[blockIdx.x];
  const int fl = it.flags;
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
  const int P = p.P, ny = p.ny, nz = p.nz, ib = p.ib, ie = p.ie;
  const long long plane_f = (long long)p.ny * p.nzp;  // field elements per x-plane
  const long long g_jk = (long long)y * p.nzp + z;   // cell offset inside a plane
  const long long plane_ax = (long long)ny * nz;     // AX psi elements per slab layer
  const int off_ax = y * nz + z;                      // AX psi offset inside a slab layer
  T *const fEX = p.fn[EX], *const fEY = p.fn[EY], *const fEZ = p.fn[EZ];
  T *const fHX = p.fn[HX], *const fHY = p.fn[HY], *const fHZ = p.fn[HZ];
  const T db = p.db, dx = p.dx, rdx = p.rdx;
  const int yc = ingrid ? y : 0, zc = ingrid ? z : 0;
  const T kye = EXACT ? p.kd[1][yc] : T(0), rkye = p.rkd[1][yc];
  const T kze = EXACT ? p.kd[2][zc] : T(0), rkze = p.rkd[2][zc];
  const T kyh = EXACT ? p.kd[4][yc] : T(0), rkyh = p.rkd[4][yc];
  const T kzh = EXACT ? p.kd[5][zc] : T(0), rkzh = p.rkd[5][zc];

  const unsigned char *tmf = static_cast<const unsigned char *>(p.tmap_f);
  const unsigned char *tmc = static_cast<const unsigned char *>(p.tmap_cb);
  auto issue = [&](int u) {  // load plane xs+u into stage u % S
    T *dst = stage + (u % S) * SB;
    unsigned long long *b = bar + (u % S);
    fence_proxy_async();
    mbar_expect_tx(b, STAGE_BYTES);
    const int xi = xs + u;
    for (int f = 0; f < 6; ++f) tma_load_3d(dst + f * BOXS, tmf + f * 128, zb, y0 - 1, xi, b);
    for (int a = 0; a < 3; ++a) tma_load_3d(dst + (6 + a) * BOXS, tmc + a * 128, zb, y0 - 1, xi, b);
  };
  // plane u lives in stage u % S and completes that stage's phase u / S
  // try_wait may suspend the thread until the phase completes, so below the
  // default bound the probes are non-blocking and the clock is read between them
  auto wait_for = [&](int k, unsigned parity, long long limit) -> bool {
    if (mbar_test_wait(bar + k, parity)) return true;
    const long long t0 = clock64();
    const bool suspend = limit >= kWaitCycles;
    for (;;) {
      if (suspend ? mbar_try_wait(bar + k, parity) : mbar_test_wait(bar + k, parity)) return true;
      if (clock64() - t0 > limit) return false;
    }
  };
  auto wait = [&](int k, unsigned parity) -> bool { return wait_for(k, parity, p.wait_cycles); };

  if (tid == 0) {
    s_abort[0] = s_abort[1] = 0;
    s_failed = 0x7fffffff;
    for (int k = 0; k < S; ++k) mbar_init(bar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    int u = 0;
    for (; u < S && u < nplanes; ++u) issue(u);
    s_issued = u;
  }
  bool ok = wait(0, 0);
  if (!ok) atomicMin(&s_failed, 0);
  bool aborted = false;

  auto march = [&](auto clean_tag) {
    constexpr bool CLEAN = decltype(clean_tag)::value;
    // ---- per-cell (j, k) classification (general march only) -----------------
    const bool jin_c = y >= p.jb && y < p.je, jin_o = y > p.jb && y < p.je;  // [jb,je) and (jb,je)
    const bool kin_c = z >= p.kb && z < p.ke, kin_o = z > p.kb && z < p.ke;  // [kb,ke) and (kb,ke)
    const bool ex_jk = CLEAN || (ingrid && jin_c && kin_c);  // Ex: j [jb,je), k [kb,ke)
    const bool ey_jk = CLEAN || (ingrid && jin_o && kin_c);  // Ey: j (jb,je), k [kb,ke)
    const bool ez_jk = CLEAN || (ingrid && jin_c && kin_o);  // Ez: j [jb,je), k (kb,ke)
    const bool hx_jk = CLEAN || (own && jin_o && kin_o);     // Hx: j (jb,je), k (kb,ke)
    const bool hy_jk = CLEAN || (own && jin_c && kin_o);     // Hy: j [jb,je), k (kb,ke)
    const bool hz_jk = CLEAN || (own && jin_o && kin_c);     // Hz: j (jb,je), k [kb,ke)
    const int ye_code = !CLEAN && (fl & kItemYSlab) && ingrid ? slab_code_e(y, p.jb, p.je, P) : -1;
    const int ze_code = !CLEAN && (fl & kItemZSlab) && ingrid ? slab_code_e(z, p.kb, p.ke, P) : -1;
    const int yh_code = !CLEAN && (fl & kItemYSlab) && own ? slab_code_h(y, p.jb, p.je, P) : -1;
    const int zh_code = !CLEAN && (fl & kItemZSlab) && own ? slab_code_h(z, p.kb, p.ke, P) : -1;
    const bool slab_yz = !CLEAN && (fl & (kItemYSlab | kItemZSlab)) != 0;
    const bool src_p = !CLEAN && (fl & kItemSrc) != 0;
    const bool src_jk = src_p && y >= p.slo[1] && y < p.shi[1] && z >= p.slo[2] && z < p.shi[2];
    const bool src_jk1 =
        src_p && p.src_field == HY && y >= p.slo[1] && y < p.shi[1] && z + 1 >= p.slo[2] && z + 1 < p.shi[2];
    const bool capt = !CLEAN && (fl & kItemPort) && own &&
                      (z == p.port_pos[0] || z == p.port_pos[1] || z == p.port_pos[0] + 1 || z == p.port_pos[1] + 1);
    const T Jn = src_p ? p.jsrc[n] : T(0);
    // psi offsets, split into a per-plane base and a per-cell part:
    // AY slabs [i][d][z] -> i*P*nz + (d*nz + z); AZ slabs [i][y][d] -> i*ny*P + (y*P + d)
    const int o_ay_e = ye_code >= 0 ? sd(ye_code) * nz + z : 0, o_az_e = ze_code >= 0 ? y * P + sd(ze_code) : 0;
    const int o_ay_h = yh_code >= 0 ? sd(yh_code) * nz + z : 0, o_az_h = zh_code >= 0 ? y * P + sd(zh_code) : 0;

    T kxe_n = EXACT ? p.kd[0][xs] : T(0), rkxe_n = p.rkd[0][xs];
    T kxh_n = EXACT ? p.kd[3][xs] : T(0), rkxh_n = p.rkd[3][xs];
    T ey_prev = T(0), ez_prev = T(0);  // new Ey, Ez of this cell at the previous plane
    int sc = 0, sn = 1 % S;            // stages of planes u and u+1
    unsigned pn = (1 / S) & 1;         // phase parity of plane u+1

    for (int u = 0; u + 1 < nplanes; ++u) {
      const int i = xs + u;
      if (ok && !(ok = wait(sn, pn))) atomicMin(&s_failed, u + 1);
      const T *const cur = stage + sc * SB;
      const T *const nxt = stage + sn * SB;
      T *const enew = sE + (u & 1) * 3 * NT;
      // ---- per-plane values (uniform) ------------------------------------------
      const bool i_c = i >= ib && i < ie, i_o = i > ib && i < ie;
      const int xe_code = slab_code_e(i, ib, ie, P);
      const int xh_code = slab_code_h(i, ib, ie, P);
      const bool edge_p = !CLEAN && ((fl & kItemEdge) || !i_o);  // per-cell range masks needed
      const T kxe = kxe_n, rkxe = rkxe_n, kxh = kxh_n, rkxh = rkxh_n;
      if (u + 2 < nplanes) {
        if (EXACT) { kxe_n = p.kd[0][i + 1]; kxh_n = p.kd[3][i + 1]; }
        rkxe_n = p.rkd[0][i + 1];
        rkxh_n = p.rkd[3][i + 1];
      }
      const bool src_i = src_p && i >= p.slo[0] && i < p.shi[0];
      const bool src_i1 = src_p && i + 1 >= p.slo[0] && i + 1 < p.shi[0];
      const long long b_ay = (long long)i * P * nz, b_az = (long long)i * ny * P;
      // ---- new E of this cell (all cells of the E box) --------------------------
      // fdtd_funcs.py:43-70 (curl), :104-110 (source), :113-188 (CPML), in that order
      const T hx0 = cur[HX * BOXS + bo], hy0 = cur[HY * BOXS + bo], hz0 = cur[HZ * BOXS + bo];
      T e0 = cur[EX * BOXS + bo], e1 = cur[EY * BOXS + bo], e2 = cur[EZ * BOXS + bo];
      const T cb0 = cur[6 * BOXS + bo], cb1 = cur[7 * BOXS + bo], cb2 = cur[8 * BOXS + bo];
      const T hy_z1 = cur[HY * BOXS + bo + 1], hy_x1 = nxt[HY * BOXS + bo];
      const T dhz_y = A::sub(cur[HZ * BOXS + bo + BZ], hz0);
      const T dhy_z = A::sub(hy_z1, hy0);
      const T dhx_z = A::sub(cur[HX * BOXS + bo + 1], hx0);
      const T dhz_x = A::sub(nxt[HZ * BOXS + bo], hz0);
      const T dhy_x = A::sub(hy_x1, hy0);
      const T dhx_y = A::sub(cur[HX * BOXS + bo + BZ], hx0);
      T nex = A::add(e0, A::mul(cb0, A::sub(A::div(dhz_y, kye, rkye), A::div(dhy_z, kze, rkze))));
      T ney = A::add(e1, A::mul(cb1, A::sub(A::div(dhx_z, kze, rkze), A::div(dhz_x, kxe, rkxe))));
      T nez = A::add(e2, A::mul(cb2, A::sub(A::div(dhy_x, kxe, rkxe), A::div(dhx_y, kye, rkye))));
      const bool mex = i_o && ex_jk, mey = i_c && ey_jk, mez = i_c && ez_jk;  // components updated here
      const bool wpsi = own && i >= x0;  // this CTA owns the cell's new psi
      if (src_i && p.src_field == EY && src_jk) ney = A::sub(ney, Jn);
      if (CLEAN) {
        if (xe_code >= 0 && i_c) {  // update_pml_ey_xinc, update_pml_ez_xinc
          const int q = sq(xe_code), sd_ = ss(xe_code);
          const long long o = (long long)sd(xe_code) * plane_ax + off_ax;
          const T vy = A::add(A::mul(p.be[q], __ldg(p.psi[EY][AX][sd_] + o)), A::div(A::mul(p.ce[q], dhz_x), dx, rdx));
          const T vz = A::add(A::mul(p.be[q], __ldg(p.psi[EZ][AX][sd_] + o)), A::div(A::mul(p.ce[q], dhy_x), dx, rdx));
          if (wpsi) {
            p.psin[EY][AX][sd_][o] = vy;
            p.psin[EZ][AX][sd_][o] = vz;
          }
          ney = A::sub(ney, A::mul(cb1, vy));
          nez = A::add(nez, A::mul(cb2, vz));
        }
        e0 = i_o ? nex : e0;
        e1 = i_c ? ney : e1;
        e2 = i_c ? nez : e2;
      } else {
        if (ok && (slab_yz || xe_code >= 0)) {
          // Hy differences seen by the CPML of Ex (along z) and Ez (along x): the
          // Hy source is applied between the E curl and the E CPML
          T dhy_zs = dhy_z, dhy_xs = dhy_x;
          if (src_p && p.src_field == HY) {
            const T jz1 = (src_i && src_jk1) ? Jn : T(0), jz0 = (src_i && src_jk) ? Jn : T(0);
            const T jx1 = (src_i1 && src_jk) ? Jn : T(0);
            dhy_zs = A::sub(A::sub(hy_z1, jz1), A::sub(hy0, jz0));
            dhy_xs = A::sub(A::sub(hy_x1, jx1), A::sub(hy0, jz0));
          }
          // all old psi values first (read-only in this launch), then the updates
          const long long b_ax = xe_code >= 0 ? (long long)sd(xe_code) * plane_ax : 0;
          const bool a_xy = mex && ye_code >= 0, a_xz = mex && ze_code >= 0, a_yx = mey && xe_code >= 0;
          const bool a_yz = mey && ze_code >= 0, a_zx = mez && xe_code >= 0, a_zy = mez && ye_code >= 0;
          const T v_xy = a_xy ? __ldg(p.psi[EX][AY][ss(ye_code)] + (b_ay + o_ay_e)) : T(0);
          const T v_xz = a_xz ? __ldg(p.psi[EX][AZ][ss(ze_code)] + (b_az + o_az_e)) : T(0);
          const T v_yx = a_yx ? __ldg(p.psi[EY][AX][ss(xe_code)] + (b_ax + off_ax)) : T(0);
          const T v_yz = a_yz ? __ldg(p.psi[EY][AZ][ss(ze_code)] + (b_az + o_az_e)) : T(0);
          const T v_zx = a_zx ? __ldg(p.psi[EZ][AX][ss(xe_code)] + (b_ax + off_ax)) : T(0);
          const T v_zy = a_zy ? __ldg(p.psi[EZ][AY][ss(ye_code)] + (b_ay + o_ay_e)) : T(0);
          if (a_xy) {  // update_pml_ex_yinc
            const int q = sq(ye_code);
            const T v = A::add(A::mul(p.be[q], v_xy), A::div(A::mul(p.ce[q], dhz_y), dx, rdx));
            if (wpsi) p.psin[EX][AY][ss(ye_code)][b_ay + o_ay_e] = v;
            nex = A::add(nex, A::mul(cb0, v));
          }
          if (a_xz) {  // update_pml_ex_zinc
            const int q = sq(ze_code);
            const T v = A::add(A::mul(p.be[q], v_xz), A::div(A::mul(p.ce[q], dhy_zs), dx, rdx));
            if (wpsi) p.psin[EX][AZ][ss(ze_code)][b_az + o_az_e] = v;
            nex = A::sub(nex, A::mul(cb0, v));
          }
          if (a_yx) {  // update_pml_ey_xinc
            const int q = sq(xe_code);
            const T v = A::add(A::mul(p.be[q], v_yx), A::div(A::mul(p.ce[q], dhz_x), dx, rdx));
            if (wpsi) p.psin[EY][AX][ss(xe_code)][b_ax + off_ax] = v;
            ney = A::sub(ney, A::mul(cb1, v));
          }
          if (a_yz) {  // update_pml_ey_zinc
            const int q = sq(ze_code);
            const T v = A::add(A::mul(p.be[q], v_yz), A::div(A::mul(p.ce[q], dhx_z), dx, rdx));
            if (wpsi) p.psin[EY][AZ][ss(ze_code)][b_az + o_az_e] = v;
            ney = A::add(ney, A::mul(cb1, v));
          }
          if (a_zx) {  // update_pml_ez_xinc
            const int q = sq(xe_code);
            const T v = A::add(A::mul(p.be[q], v_zx), A::div(A::mul(p.ce[q], dhy_xs), dx, rdx));
            if (wpsi) p.psin[EZ][AX][ss(xe_code)][b_ax + off_ax] = v;
            nez = A::add(nez, A::mul(cb2, v));
          }
          if (a_zy) {  // update_pml_ez_yinc
            const int q = sq(ye_code);
            const T v = A::add(A::mul(p.be[q], v_zy), A::div(A::mul(p.ce[q], dhx_y), dx, rdx));
            if (wpsi) p.psin[EZ][AY][ss(ye_code)][b_ay + o_ay_e] = v;
            nez = A::sub(nez, A::mul(cb2, v));
          }
        }
        if (edge_p) {
          e0 = mex ? nex : e0;
          e1 = mey ? ney : e1;
          e2 = mez ? nez : e2;
        } else {
          e0 = nex;
          e1 = ney;
          e2 = nez;
        }
      }
      enew[tid] = e0;
      enew[NT + tid] = e1;
      enew[2 * NT + tid] = e2;
      if (!ok) s_abort[u & 1] = 1;
      __syncthreads();  // new E of the tile visible; stage sc no longer read
      if (s_abort[u & 1]) {
        aborted = true;
        break;
      }
      if (tid == 0 && u + S < nplanes) {
        issue(u + S);  // into stage sc
        s_issued = u + S + 1;
      }
      // ---- new H of owned cells; store E and H ------------------------------------
      // fdtd_funcs.py:73-100 (curl), :83-90 (Hy source before update_hy), :191-266 (CPML)
      if (i >= x0) {
        // halo cells (row 0 / column 0 of the E box) compute too and store nothing
        const T dey_z = A::sub(e1, enew[NT + tid - 1]);
        const T dez_y = A::sub(e2, enew[2 * NT + tid - TBZ]);
        const T dez_x = A::sub(e2, ez_prev);
        const T dex_z = A::sub(e0, enew[tid - 1]);
        const T dex_y = A::sub(e0, enew[tid - TBZ]);
        const T dey_x = A::sub(e1, ey_prev);
        T hy_s = hy0;
        if (src_i && p.src_field == HY && src_jk) hy_s = A::sub(hy_s, Jn);
        T nhx = A::add(hx0, A::mul(db, A::sub(A::div(dey_z, kzh, rkzh), A::div(dez_y, kyh, rkyh))));
        T nhy = A::add(hy_s, A::mul(db, A::sub(A::div(dez_x, kxh, rkxh), A::div(dex_z, kzh, rkzh))));
        T nhz = A::add(hz0, A::mul(db, A::sub(A::div(dex_y, kyh, rkyh), A::div(dey_x, kxh, rkxh))));
        const bool mhx = own && i_c && hx_jk, mhy = own && i_o && hy_jk, mhz = own && i_o && hz_jk;
        T h0v, h1v, h2v;
        if (CLEAN) {
          if (xh_code >= 0 && i_o && own) {  // update_pml_hy_xinc, update_pml_hz_xinc (in place)
            const int q = sq(xh_code), sd_ = ss(xh_code);
            const long long o = (long long)sd(xh_code) * plane_ax + off_ax;
            T *const py = p.psi[HY][AX][sd_] + o;
            T *const pz = p.psi[HZ][AX][sd_] + o;
            const T oy = *py, oz = *pz;
            const T vy = A::add(A::mul(p.bh[q], oy), A::div(A::mul(p.ch[q], dez_x), dx, rdx));
            const T vz = A::add(A::mul(p.bh[q], oz), A::div(A::mul(p.ch[q], dey_x), dx, rdx));
            *py = vy;
            *pz = vz;
            nhy = A::add(nhy, A::mul(db, vy));
            nhz = A::sub(nhz, A::mul(db, vz));
          }
          h0v = i_c ? nhx : hx0;
          h1v = i_o ? nhy : hy0;
          h2v = i_o ? nhz : hz0;
        } else {
          if (slab_yz || xh_code >= 0) {
            // H psi is updated in place, each element by its own cell only: loads first
            const long long b_ax = xh_code >= 0 ? (long long)sd(xh_code) * plane_ax : 0;
            const bool a_xy = mhx && yh_code >= 0, a_xz = mhx && zh_code >= 0, a_yx = mhy && xh_code >= 0;
            const bool a_yz = mhy && zh_code >= 0, a_zx = mhz && xh_code >= 0, a_zy = mhz && yh_code >= 0;
            T *const q_xy = p.psi[HX][AY][a_xy ? ss(yh_code) : 0] + (b_ay + o_ay_h);
            T *const q_xz = p.psi[HX][AZ][a_xz ? ss(zh_code) : 0] + (b_az + o_az_h);
            T *const q_yx = p.psi[HY][AX][a_yx ? ss(xh_code) : 0] + (b_ax + off_ax);
            T *const q_yz = p.psi[HY][AZ][a_yz ? ss(zh_code) : 0] + (b_az + o_az_h);
            T *const q_zx = p.psi[HZ][AX][a_zx ? ss(xh_code) : 0] + (b_ax + off_ax);
            T *const q_zy = p.psi[HZ][AY][a_zy ? ss(yh_code) : 0] + (b_ay + o_ay_h);
            const T v_xy = a_xy ? *q_xy : T(0), v_xz = a_xz ? *q_xz : T(0), v_yx = a_yx ? *q_yx : T(0);
            const T v_yz = a_yz ? *q_yz : T(0), v_zx = a_zx ? *q_zx : T(0), v_zy = a_zy ? *q_zy : T(0);
            if (a_xy) {  // update_pml_hx_yinc
              const int q = sq(yh_code);
              const T v = A::add(A::mul(p.bh[q], v_xy), A::div(A::mul(p.ch[q], dez_y), dx, rdx));
              *q_xy = v;
              nhx = A::sub(nhx, A::mul(db, v));
            }
            if (a_xz) {  // update_pml_hx_zinc
              const int q = sq(zh_code);
              const T v = A::add(A::mul(p.bh[q], v_xz), A::div(A::mul(p.ch[q], dey_z), dx, rdx));
              *q_xz = v;
              nhx = A::add(nhx, A::mul(db, v));
            }
            if (a_yx) {  // update_pml_hy_xinc
              const int q = sq(xh_code);
              const T v = A::add(A::mul(p.bh[q], v_yx), A::div(A::mul(p.ch[q], dez_x), dx, rdx));
              *q_yx = v;
              nhy = A::add(nhy, A::mul(db, v));
            }
            if (a_yz) {  // update_pml_hy_zinc
              const int q = sq(zh_code);
              const T v = A::add(A::mul(p.bh[q], v_yz), A::div(A::mul(p.ch[q], dex_z), dx, rdx));
              *q_yz = v;
              nhy = A::sub(nhy, A::mul(db, v));
            }
            if (a_zx) {  // update_pml_hz_xinc
              const int q = sq(xh_code);
              const T v = A::add(A::mul(p.bh[q], v_zx), A::div(A::mul(p.ch[q], dey_x), dx, rdx));
              *q_zx = v;
              nhz = A::sub(nhz, A::mul(db, v));
            }
            if (a_zy) {  // update_pml_hz_yinc
              const int q = sq(yh_code);
              const T v = A::add(A::mul(p.bh[q], v_zy), A::div(A::mul(p.ch[q], dex_y), dx, rdx));
              *q_zy = v;
              nhz = A::add(nhz, A::mul(db, v));
            }
          }
          if (edge_p) {
            h0v = mhx ? nhx : hx0;
            h1v = mhy ? nhy : hy0;
            h2v = mhz ? nhz : hz0;
          } else {
            h0v = nhx;
            h1v = nhy;
            h2v = nhz;
          }
          if (capt) {
            const T ev[3] = {e0, e1, e2}, hv[3] = {h0v, h1v, h2v};
            const int me = (mex ? 1 : 0) | (mey ? 2 : 0) | (mez ? 4 : 0);
            const int mh = (mhx ? 1 : 0) | (mhy ? 2 : 0) | (mhz ? 4 : 0);
            y3_capture_e(p, s, i, y, z, me, ev);
            y3_capture_h(p, s, i, y, z, mh, hv);
          }
        }
        if (own) {
          const long long g = (long long)i * plane_f + g_jk;
          fEX[g] = e0;
          fEY[g] = e1;
          fEZ[g] = e2;
          fHX[g] = h0v;
          fHY[g] = h1v;
          fHZ[g] = h2v;
        }
      }
      ey_prev = e1;
      ez_prev = e2;
      sc = sn;
      if (++sn == S) {
        sn = 0;
        pn ^= 1u;
      }
    }
  };
  if (fl == 0)
    march(std::true_type{});
  else
    march(std::false_type{});

  if (aborted && tid == 0) {
    atomicExch(p.state + 1, 1);  // reported to the host by oidt_job_sync
    // copies issued after the failed one: bounded wait so none lands after exit
    for (int v = s_failed; v < s_issued; ++v) (void)wait_for(v % S, (unsigned)((v / S) & 1), kWaitCycles);
  }
}

}  // namespace oidt
