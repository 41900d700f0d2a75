// tile2d.cuh -- 2D TM / TE time steps, temporally blocked in tiles.
//
// A 2D job of the served sizes (a few hundred x a few hundred cells) is too
// small to fill the GPU, so with one launch per half-step its step time is
// launch latency.  Here the grid advances in sub-blocks of up to `halo` steps,
// a launch covering one sub-block or a whole ring block of them:
//
// * The grid is cut into tiles, one block each.  Block (bi, bj) owns the
//   cells [oi0, oi1) x [oj0, oj1) and also computes `halo` cells on every side
//   of them ([wi0, wi1) x [wj0, wj1), clipped to the grid).  A step's E half
//   reads H at (i + 1, j) and (i, j + 1), its H half E at (i - 1, j) and
//   (i, j - 1), so after s steps the cells a block holds are exact s cells
//   inside the held tile's edges (and up to the grid's edges, where there is
//   nothing to read): after cnt <= halo steps the owned cells are exact.
// * A held tile has at most kTileThreads cells, one per thread.  A thread
//   works out its cell's update conditions, CPML slab coefficients and dt/eps
//   values once per launch and keeps them in registers, and so its cell's
//   three field values and CPML psi values through a sub-block of up to
//   `halo` steps.  Shared memory holds the tile's fields only for the
//   neighbours' reads (each value written once per half-step by its cell's
//   thread), the CPML coefficient tables, and the kappa dx divisors with
//   their reciprocals for the tile's rows and columns; __syncthreads
//   separates the half-steps.
// * Fields and psi are double-buffered: sub-block b reads the state of
//   buffer par ^ (b & 1) and writes its owned cells to the other, so blocks
//   loading halo cells never see cells another block has already advanced.
// * A launch of one sub-block (cnt <= halo) needs no other synchronisation:
//   a grid with more tiles than SMs simply runs in waves.  A launch of
//   several sub-blocks is cooperative (all tiles resident at once): before
//   sub-block b > 0 a block waits until each of its (up to 8) neighbour tiles
//   has published, through its counter in `epoch` (release / acquire), that
//   it finished sub-block b - 1 -- its owned cells written, its reads of the
//   buffer this block writes next done.  Halo width <= tile extent, so no
//   other tile's cells are read.  The wait is bounded (p.wait_cycles); on
//   expiry the block records state[1] = 3 and goes on.  Between sub-blocks
//   only what other tiles read crosses global memory: a tile stores its owned
//   cells within `halo` of its edges and reloads its halo cells; the other
//   owned cells stay in registers (and are stored after the last sub-block).
//
// Per cell the arithmetic is that of kernels.cuh's tm2_e_cell / tm2_h_cell /
// te2_e_cell / te2_h_cell (the reference's fdtd_funcs.py of FDTD_2D_TM and
// FDTD_2D_TE, lines 43-124, in its launch order), operation for operation, so
// EXACT runs equal the reference and the oracle bit for bit; halo cells are
// computed with the same operations and never written back.
#pragma once

#include "kernels.cuh"

namespace oidt {

constexpr int kTileThreads = 1024;  // also the most cells a held tile has
constexpr int kTileHaloMax = 8;     // steps per sub-block at most

struct TileArgs {
  int s0;      // ring slot of the launch's first step
  int cnt;     // steps of this launch (more than halo: a cooperative launch of several sub-blocks)
  int ti, tj;  // owned tile extent: rows (x), columns (y)
  int gj;      // tiles along y
  int halo;    // cells computed on each side of the owned tile; steps per sub-block
  int *epoch;  // per tile: sub-blocks completed (cooperative launches)
};

// Shared memory of a block: the tile's three fields (kTileThreads cells each),
// the CPML coefficient tables be, ce, bh, ch (P each), and per held row (at
// most rows) kd0, 1/kd0, kd3, 1/kd3, per held column (at most cols) kd1,
// 1/kd1, kd4, 1/kd4 (the kappa dx arrays: E x, H x, E y, H y).
inline size_t tile2d_smem(int esz, int P, int rows, int cols) {
  return (3 * (size_t)kTileThreads + 4 * (size_t)P + 4 * (size_t)rows + 4 * (size_t)cols) * esz;
}

// Cell flags.  TM: E1 = Ez update, H1 = Hx, H2 = Hy; TE: E1 = Ex, E2 = Ey,
// H1 = Hz.  XE / YE / XH / YH: the cell is in the E / H x- / y-slab of the
// CPML.  CE0 / CE1, CH0 / CH1: the cell's E / H value is captured into the
// ring for port 0 / 1 (E slot 0 and H slot 1 at x = port, H slot 2 at
// x = port + 1).
enum : unsigned {
  kE1 = 1u, kE2 = 2u, kH1 = 4u, kH2 = 8u, kSrc = 16u, kXE = 32u, kYE = 64u, kXH = 128u, kYH = 256u,
  kCE0 = 512u, kCE1 = 1024u, kCH0 = 2048u, kCH1 = 4096u, kOwn = 8192u, kBand = 16384u
};

template <typename T, bool EXACT, int MODE>
__global__ void __launch_bounds__(kTileThreads, 1) k_2d_tile(Params<T> p, TileArgs a) {
  using A = Ar<T, EXACT>;
  constexpr bool TM = MODE == OIDT_MODE_TM2;
  // fields f0, f1 (E in TE, H in TM), f2 (H); the fields carrying each psi array
  constexpr int FA = TM ? EZ : EX, FB = TM ? HX : EY, FC = TM ? HY : HZ;
  constexpr int EXS = TM ? EZ : EY, EYS = TM ? EZ : EX, HXS = TM ? HY : HZ, HYS = TM ? HX : HZ;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *const F0 = reinterpret_cast<T *>(smem_raw), *const F1 = F0 + kTileThreads, *const F2 = F1 + kTileThreads;
  T *const BE = F2 + kTileThreads, *const CE = BE + p.P, *const BH = CE + p.P, *const CH = BH + p.P;
  // kd, 1/kd tables (one array each, consecutive columns in consecutive banks): rows kd0 1/kd0 kd3 1/kd3,
  // columns kd1 1/kd1 kd4 1/kd4
  const int RM = a.ti + 2 * a.halo, CM = a.tj + 2 * a.halo;
  T *const KR = CH + p.P, *const KC = KR + 4 * RM;
  const int nx = p.nx, ny = p.ny, P = p.P, H = a.halo;
  const int bi = (int)blockIdx.x / a.gj, bj = (int)blockIdx.x - bi * a.gj;
  const int oi0 = bi * a.ti, oi1 = min(nx, oi0 + a.ti), oj0 = bj * a.tj, oj1 = min(ny, oj0 + a.tj);
  const int wi0 = max(0, oi0 - H), wi1 = min(nx, oi1 + H), wj0 = max(0, oj0 - H), wj1 = min(ny, oj1 + H);
  const int nrow = wi1 - wi0, ncol = wj1 - wj0;
  const int t = threadIdx.x;
  const bool act = t < nrow * ncol;
  const int li = act ? t / ncol : 0, lj = act ? t - li * ncol : 0, i = wi0 + li, j = wj0 + lj;
  const int g = i * ny + j;  // the cell in the [nx][ny] arrays (2^31 cells at most)
  // ---- the cell's constants ------------------------------------------------------------
  unsigned fl = 0;
  int qE = 0, qH = 0;  // slab coefficient indices + 1: x slab in bits 0-15, y slab in bits 16-31
  T cbA = T(0), cbB = T(0);  // dt/eps of the cell's E components
  int capE[2] = {0, 0}, capH[2] = {0, 0};  // ring offsets of the cell's captures within a slot, per port
  // psi offsets of the cell in its slab arrays (x slab [P][ny], y slab [nx][P]) and their sides
  int oxE = 0, oyE = 0, oxH = 0, oyH = 0, sides = 0;  // sides: bit 0 x E, 1 y E, 2 x H, 3 y H
  // this thread's entries of the coefficient and kappa dx tables, loaded first so that
  // their latency overlaps the cell's own loads (leftovers past kTileThreads below)
  const int nk = 4 * (nrow + ncol);
  auto co_src = [&](int u) { return __ldg((u < P ? p.be : u < 2 * P ? p.ce : u < 3 * P ? p.bh : p.ch) + u % P); };
  auto k_src = [&](int u, int &dst) {  // rows kd0 1/kd0 kd3 1/kd3, then columns kd1 1/kd1 kd4 1/kd4
    const bool row = u < 4 * nrow;
    const int v = row ? u : u - 4 * nrow, n = row ? nrow : ncol, c = v / n, r = v - c * n;
    const int a_ = row ? (c < 2 ? 0 : 3) : (c < 2 ? 1 : 4);
    dst = row ? c * RM + r : 4 * RM + c * CM + r;
    return __ldg((c & 1 ? p.rkd[a_] : p.kd[a_]) + (row ? wi0 : wj0) + r);
  };
  int kdst = 0;
  const T vco = t < 4 * P ? co_src(t) : T(0);
  const T vk = t < nk ? k_src(t, kdst) : T(0);
  if (act) {
    int d, side, q;
    if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {
      oxE = d * ny + j;
      sides |= side;
      fl |= kXE;
      qE |= q + 1;
    }
    if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {
      oyE = i * P + d;
      sides |= side << 1;
      fl |= kYE;
      qE |= (q + 1) << 16;
    }
    if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {
      oxH = d * ny + j;
      sides |= side << 2;
      fl |= kXH;
      qH |= q + 1;
    }
    if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {
      oyH = i * P + d;
      sides |= side << 3;
      fl |= kYH;
      qH |= (q + 1) << 16;
    }
    // neighbours at (i + 1, j), (i, j + 1) [E] and (i - 1, j), (i, j - 1) [H] exist in
    // the tile except on its edges, whose cells are halo cells when not on the grid's edge
    const bool up = li + 1 < nrow, right = lj + 1 < ncol, down = li > 0, left = lj > 0;
    const bool own = i >= oi0 && i < oi1 && j >= oj0 && j < oj1;
    if (own) fl |= kOwn;
    if (own && (i - oi0 < H || oi1 - i <= H || j - oj0 < H || oj1 - j <= H)) fl |= kBand;  // read by neighbour tiles
    if (TM) {
      if (i >= p.ib && i < p.ie && j >= p.jb && j < p.je && up && right) fl |= kE1;   // update_ez :44-49
      if (i >= p.ib && i < p.ie && j > p.jb && j < p.je && left) fl |= kH1;          // update_hx :53-58
      if (i > p.ib && i < p.ie && j >= p.jb && j < p.je && down) fl |= kH2;          // update_hy :62-67
      if (in_src(p, EZ, i, j, 0)) fl |= kSrc;
      cbA = __ldg(p.cb[2] + g);
    } else {
      if (i > p.ib && i < p.ie && j >= p.jb && j < p.je && right) fl |= kE1;         // update_ex :43-49
      if (i >= p.ib && i < p.ie && j > p.jb && j < p.je && up) fl |= kE2;            // update_ey :52-58
      if (i > p.ib && i < p.ie && j > p.jb && j < p.je && down && left) fl |= kH1;   // update_hz :61-67
      if (in_src(p, HZ, i, j, 0)) fl |= kSrc;
      cbA = __ldg(p.cb[0] + g);
      cbB = __ldg(p.cb[1] + g);
    }
    // ring captures of an owned cell on a port plane (where the update of the captured component runs)
    for (int port = 0; port < 2 && own; ++port) {
      const int x = p.port_pos[port];
      if (i == x && (fl & (TM ? kE1 : kE2))) {
        fl |= kCE0 << port;
        capE[port] = (port * p.nslot + 0) * (int)p.plane + j;
      }
      if ((i == x || i == x + 1) && (fl & (TM ? kH2 : kH1))) {
        fl |= kCH0 << port;
        capH[port] = (port * p.nslot + (i == x ? 1 : 2)) * (int)p.plane + j;
      }
    }
  }
  if (t < 4 * P) BE[t] = vco;  // the CPML coefficients be ce bh ch, and the kappa dx tables
  if (t < nk) KR[kdst] = vk;
  for (int u = t + kTileThreads; u < 4 * P; u += kTileThreads) BE[u] = co_src(u);
  for (int u = t + kTileThreads; u < nk; u += kTileThreads) {
    int dst;
    const T x = k_src(u, dst);
    KR[dst] = x;
  }
  const T *const kr = KR + li, *const kc = KC + lj;  // kr[0, RM, 2 RM, 3 RM]: kd0 1/kd0 kd3 1/kd3; kc likewise
  const T db = p.db;
  const long long cstride = 2LL * p.nslot * p.plane;  // ring slot pitch
  const int nsub = (a.cnt + H - 1) / H;
  pdl_wait();  // the previous launch's state is complete (and visible) from here on
  const int n0 = p.state[0] + a.s0;
  const int e0 = nsub > 1 ? a.epoch[blockIdx.x] : 0;  // equal for every tile at launch
  T f0 = T(0), f1 = T(0), f2 = T(0), xe = T(0), ye = T(0), xh = T(0), yh = T(0);  // the cell's values
  for (int sb = 0; sb < nsub; ++sb) {
    T **rf = (sb & 1) ? p.fn : p.f;  // buffers read and written in this sub-block
    T **wf = (sb & 1) ? p.f : p.fn;
    T *(*rp)[3][2] = (sb & 1) ? p.psin : p.psi;
    T *(*wp)[3][2] = (sb & 1) ? p.psi : p.psin;
    if (sb > 0) {  // the neighbour tiles have finished sub-block sb - 1
      if (t < 9 && t != 4) {
        const int nbi = bi + t / 3 - 1, nbj = bj + t % 3 - 1;
        const int gi = (nx + a.ti - 1) / a.ti;
        if (nbi >= 0 && nbi < gi && nbj >= 0 && nbj < a.gj) {
          const int *ep = a.epoch + nbi * a.gj + nbj;
          const long long t0 = clock64();
          while (ld_acquire(ep) < e0 + sb) {
            if (clock64() - t0 > p.wait_cycles) {
              atomicExch(p.state + 1, 3);  // reported to the host by oidt_job_sync
              break;
            }
            if (ld_acquire(p.state + 1) != 0) break;  // an earlier wait expired: stop waiting
          }
        }
      }
      __syncthreads();
    }
    if (act && (sb == 0 || !(fl & kOwn))) {  // the held tile of the buffer read (L2: other blocks wrote it)
      f0 = __ldcg(rf[FA] + g);
      f1 = __ldcg(rf[FB] + g);
      f2 = __ldcg(rf[FC] + g);
      F0[t] = f0;
      F1[t] = f1;
      F2[t] = f2;
      if (fl & kXE) xe = __ldcg(rp[EXS][AX][sides & 1] + oxE);
      if (fl & kYE) ye = __ldcg(rp[EYS][AY][(sides >> 1) & 1] + oyE);
      if (fl & kXH) xh = __ldcg(rp[HXS][AX][(sides >> 2) & 1] + oxH);
      if (fl & kYH) yh = __ldcg(rp[HYS][AY][(sides >> 3) & 1] + oyH);
    }
    __syncthreads();
    const int s1 = min(a.cnt, (sb + 1) * H);
    for (int s = sb * H; s < s1; ++s) {
      T *const ring = p.ring + (a.s0 + s) * cstride;  // the step's ring slot
      // ---- E half-step ------------------------------------------------------------------
      if (TM) {
        if (fl & kE1) {  // update_ez :44-49
          const T dhy = A::sub(F2[t + ncol], f2);
          const T dhx = A::sub(F1[t + 1], f1);
          T e = A::add(f0, A::mul(cbA, A::sub(A::div(dhy, kr[0], kr[RM]), A::div(dhx, kc[0], kc[CM]))));
          if (fl & kSrc) e = A::sub(e, __ldg(p.jsrc + n0 + s));  // update_source :71-76
          if (fl & kXE) {                                        // update_pml_ez_xinc :80-88
            const int q = (qE & 0xffff) - 1;
            xe = A::add(A::mul(BE[q], xe), A::div(A::mul(CE[q], dhy), p.dx, p.rdx));
            e = A::add(e, A::mul(cbA, xe));
          }
          if (fl & kYE) {                                        // update_pml_ez_yinc :92-100
            const int q = (qE >> 16) - 1;
            ye = A::add(A::mul(BE[q], ye), A::div(A::mul(CE[q], dhx), p.dx, p.rdx));
            e = A::sub(e, A::mul(cbA, ye));
          }
          f0 = e;
          F0[t] = e;
          if (fl & kCE0) ring[capE[0]] = e;
          if (fl & kCE1) ring[capE[1]] = e;
        }
      } else {
        if (fl & kE1) {  // update_ex :43-49
          const T dhz = A::sub(F2[t + 1], f2);
          T e = A::add(f0, A::div(A::mul(cbA, dhz), kc[0], kc[CM]));
          if (fl & kYE) {                                        // update_pml_ex_yinc :79-87
            const int q = (qE >> 16) - 1;
            ye = A::add(A::mul(BE[q], ye), A::div(A::mul(CE[q], dhz), p.dx, p.rdx));
            e = A::add(e, A::mul(cbA, ye));
          }
          f0 = e;
          F0[t] = e;
        }
        if (fl & kE2) {  // update_ey :52-58
          const T hz1 = F2[t + ncol];
          T e = A::add(f1, A::div(A::mul(cbB, A::sub(f2, hz1)), kr[0], kr[RM]));
          if (fl & kXE) {                                        // update_pml_ey_xinc :91-99
            const int q = (qE & 0xffff) - 1;
            xe = A::add(A::mul(BE[q], xe), A::div(A::mul(CE[q], A::sub(hz1, f2)), p.dx, p.rdx));
            e = A::sub(e, A::mul(cbB, xe));
          }
          f1 = e;
          F1[t] = e;
          if (fl & kCE0) ring[capE[0]] = e;
          if (fl & kCE1) ring[capE[1]] = e;
        }
      }
      __syncthreads();
      // ---- H half-step ------------------------------------------------------------------
      if (TM) {
        if (fl & kH1) {  // update_hx :53-58
          const T ezm = F0[t - 1];
          T h = A::add(f1, A::div(A::mul(db, A::sub(ezm, f0)), kc[2 * CM], kc[3 * CM]));
          if (fl & kYH) {                                        // update_pml_hx_yinc :104-112
            const int q = (qH >> 16) - 1;
            yh = A::add(A::mul(BH[q], yh), A::div(A::mul(CH[q], A::sub(f0, ezm)), p.dx, p.rdx));
            h = A::sub(h, A::mul(db, yh));
          }
          f1 = h;
          F1[t] = h;
        }
        if (fl & kH2) {  // update_hy :62-67
          const T dez = A::sub(f0, F0[t - ncol]);
          T h = A::add(f2, A::div(A::mul(db, dez), kr[2 * RM], kr[3 * RM]));
          if (fl & kXH) {                                        // update_pml_hy_xinc :116-124
            const int q = (qH & 0xffff) - 1;
            xh = A::add(A::mul(BH[q], xh), A::div(A::mul(CH[q], dez), p.dx, p.rdx));
            h = A::add(h, A::mul(db, xh));
          }
          f2 = h;
          F2[t] = h;
          if (fl & kCH0) ring[capH[0]] = h;
          if (fl & kCH1) ring[capH[1]] = h;
        }
      } else {
        if (fl & kH1) {  // update_hz :61-67
          const T dex = A::sub(f0, F0[t - 1]);
          const T dey = A::sub(f1, F1[t - ncol]);
          T h = A::add(f2, A::mul(db, A::sub(A::div(dex, kc[2 * CM], kc[3 * CM]), A::div(dey, kr[2 * RM], kr[3 * RM]))));
          if (fl & kSrc) h = A::sub(h, __ldg(p.jsrc + n0 + s));  // source after update_hz
          if (fl & kXH) {                                        // update_pml_hz_xinc :103-111
            const int q = (qH & 0xffff) - 1;
            xh = A::add(A::mul(BH[q], xh), A::div(A::mul(CH[q], dey), p.dx, p.rdx));
            h = A::sub(h, A::mul(db, xh));
          }
          if (fl & kYH) {                                        // update_pml_hz_yinc :115-123
            const int q = (qH >> 16) - 1;
            yh = A::add(A::mul(BH[q], yh), A::div(A::mul(CH[q], dex), p.dx, p.rdx));
            h = A::add(h, A::mul(db, yh));
          }
          f2 = h;
          F2[t] = h;
          if (fl & kCH0) ring[capH[0]] = h;
          if (fl & kCH1) ring[capH[1]] = h;
        }
      }
      __syncthreads();
    }
    // ---- owned cells to the buffer written (before the last sub-block: those other tiles read)
    if ((fl & kOwn) && (sb == nsub - 1 || (fl & kBand))) {
      wf[FA][g] = f0;
      wf[FB][g] = f1;
      wf[FC][g] = f2;
      if (fl & kXE) wp[EXS][AX][sides & 1][oxE] = xe;
      if (fl & kYE) wp[EYS][AY][(sides >> 1) & 1][oyE] = ye;
      if (fl & kXH) wp[HXS][AX][(sides >> 2) & 1][oxH] = xh;
      if (fl & kYH) wp[HYS][AY][(sides >> 3) & 1][oyH] = yh;
    }
    if (nsub > 1) {  // publish: this tile finished sub-block sb (the barrier orders every
      __syncthreads();  // thread's stores before thread 0's fence, which is cumulative)
      if (t == 0) {
        __threadfence();
        st_release(a.epoch + blockIdx.x, e0 + sb + 1);
      }
    }
  }
}

}  // namespace oidt
