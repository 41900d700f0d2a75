// vec3d.cuh -- 3D Yee E and H half-steps, vector form.
//
// One launch per half-step, in two roles over one x-plane per grid row:
//
// * vector role: the z-clean cells, k in [kz0, kz1) = [kb + P, ke - P)
//   rounded inward to multiples of 4, where no cell is in a z slab or on the
//   rim.  A thread owns four consecutive cells along z (the guide axis,
//   contiguous in memory) of one (i, j) row.  Rows are padded to nzp (a
//   multiple of 4 cells) and every sub-buffer starts on a 256-byte boundary,
//   so each field, dt/eps grid, z kappa array and x/y-slab psi row moves in
//   16-byte accesses (float4, or two double2 in float64).  The x-slab terms
//   are uniform over a block and the y-slab terms over a row, and so are the
//   component update ranges (only i = ib and j = jb leave a component out):
//   no per-cell test runs in this role.  A plane is a flat list of (row,
//   four-cell group) pairs, so no lane idles whatever nz is.
// * edge role: every other four-cell group (the z slabs, the rim and the row
//   padding: 9 % of the cells of a 256-cell guide with a 10-cell CPML), with
//   each component's update range tested per cell and the z-slab psi moved
//   per group in rows padded to whole groups.
//
// Per cell the arithmetic is the sequence of kernels.cuh's y3_e_compute /
// y3_h_compute (the reference's fdtd_funcs.py:43-266 in its launch order):
// curl update, soft source, then the CPML terms of the x, y and z slabs.  With
// EXACT arithmetic every operation is the reference's IEEE operation, so
// float64 runs equal the reference and the oracle bit for bit.
//
// Cells next to the source box take the general per-cell path (y3_e_cell /
// y3_h_cell) in both roles of the E half-step: with the 'TM' source (Hy) the
// reference subtracts J from Hy between the E curl and the E CPML kernels, so
// the x-slab term of Ez and the z-slab term of Ex read Hy - J there.
#pragma once
#include "kernels.cuh"

namespace oidt {

constexpr int kVecThreads = 128;
// Six resident blocks per SM in FP32 (at most 80 registers a thread): the
// vector role's loads in flight come from occupancy, and the edge role's
// longer code would otherwise raise the whole kernel's register count
// (measured: with six blocks C2 73.9 us and a 384 x 384 x 256 grid 0.612 ms
// per step, against 83.6 and 0.694 with the compiler's own 96-107 registers).
// FP64 values take two registers each: three blocks (170 registers) keep the
// FP64 kernels from spilling.  The E half-step runs seven blocks (72
// registers, a few spills to L1): C2 71.6 against 72.8 us per step; eight
// blocks (64 registers) spill more and lose (76.1).
constexpr int kVecBlocksPerSM = 6;
constexpr int kVecBlocksPerSME = 7;

template <typename T> struct V4 { T v[4]; };

// read-only data of this launch (non-coherent path)
__device__ __forceinline__ void ld4(V4<float> &a, const float *p) {
  const float4 x = __ldg(reinterpret_cast<const float4 *>(p));
  a.v[0] = x.x; a.v[1] = x.y; a.v[2] = x.z; a.v[3] = x.w;
}
__device__ __forceinline__ void ld4(V4<double> &a, const double *p) {
  const double2 x = __ldg(reinterpret_cast<const double2 *>(p)), y = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  a.v[0] = x.x; a.v[1] = x.y; a.v[2] = y.x; a.v[3] = y.y;
}
// E in an H update: L2 only (CG) where the same launch may have written E on
// another SM, whose writes an SM's L1 does not see; the read-only path otherwise
template <bool CG> __device__ __forceinline__ void ld4e(V4<float> &a, const float *p) {
  if (!CG) return ld4(a, p);
  const float4 x = __ldcg(reinterpret_cast<const float4 *>(p));
  a.v[0] = x.x; a.v[1] = x.y; a.v[2] = x.z; a.v[3] = x.w;
}
template <bool CG> __device__ __forceinline__ void ld4e(V4<double> &a, const double *p) {
  if (!CG) return ld4(a, p);
  const double2 x = __ldcg(reinterpret_cast<const double2 *>(p)), y = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
  a.v[0] = x.x; a.v[1] = x.y; a.v[2] = y.x; a.v[3] = y.y;
}
// data this launch also writes (each element only by the thread reading it)
__device__ __forceinline__ void ldw4(V4<float> &a, const float *p) {
  const float4 x = *reinterpret_cast<const float4 *>(p);
  a.v[0] = x.x; a.v[1] = x.y; a.v[2] = x.z; a.v[3] = x.w;
}
__device__ __forceinline__ void ldw4(V4<double> &a, const double *p) {
  const double2 x = reinterpret_cast<const double2 *>(p)[0], y = reinterpret_cast<const double2 *>(p)[1];
  a.v[0] = x.x; a.v[1] = x.y; a.v[2] = y.x; a.v[3] = y.y;
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double (&v)[4]) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}

// dt/eps of four cells: from the material index and its table (one byte per
// cell, the table entries read through L1) or from the three grids.
__device__ __forceinline__ void tab_entry(const float *t, unsigned q, float &a, float &b, float &c) {
  const float4 e = __ldg(reinterpret_cast<const float4 *>(t) + q);
  a = e.x; b = e.y; c = e.z;
}
__device__ __forceinline__ void tab_entry(const double *t, unsigned q, double &a, double &b, double &c) {
  const double2 e = __ldg(reinterpret_cast<const double2 *>(t) + 2 * q), f = __ldg(reinterpret_cast<const double2 *>(t) + 2 * q + 1);
  a = e.x; b = e.y; c = f.x;
}
template <typename T>
__device__ __forceinline__ void load_cb(const Params<T> &p, long long bi, int o, V4<T> &C0, V4<T> &C1, V4<T> &C2) {
  if (p.mat) {
    const uchar4 m = __ldg(reinterpret_cast<const uchar4 *>(p.mat + bi + o));
    tab_entry(p.mtab, m.x, C0.v[0], C1.v[0], C2.v[0]);
    tab_entry(p.mtab, m.y, C0.v[1], C1.v[1], C2.v[1]);
    tab_entry(p.mtab, m.z, C0.v[2], C1.v[2], C2.v[2]);
    tab_entry(p.mtab, m.w, C0.v[3], C1.v[3], C2.v[3]);
  } else {
    ld4(C0, p.cb[0] + bi + o);
    ld4(C1, p.cb[1] + bi + o);
    ld4(C2, p.cb[2] + bi + o);
  }
}

// Prefetch (into L2) of the CPML psi lines a group reads after its curl (its
// x- and y-slab rows and, in the edge role, its z-slab row), issued before the
// field loads so that the late loads find the lines on chip.  A prefetch holds
// no register; the addresses are those the group loads later.  Used by both
// roles of the H half-step and by the E half-step's edge role: in the E
// vector role it measured slower on large grids (the 384 x 384 x 256 E
// half-step 301 against 286 us), elsewhere faster (C2 step 68.1 against
// 69.8 us).
__device__ __forceinline__ void prefetch_line(const void *a) { asm volatile("prefetch.global.L2 [%0];" ::"l"(a)); }
template <typename T, bool HALF_H>
__device__ __forceinline__ void psi_prefetch(const Params<T> &p, int i, int j, int k0, bool zslab) {
  constexpr int FX0 = HALF_H ? HY : EY, FX1 = HALF_H ? HZ : EZ, FY0 = HALF_H ? HX : EX, FY1 = HALF_H ? HZ : EZ;
  constexpr int FZ0 = HALF_H ? HX : EX, FZ1 = HALF_H ? HY : EY;
  const int P = p.P;
  int d, side;
  if ((HALF_H ? h_slab(i, p.ib, p.ie, P, d, side) : e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {
    const long long oa = ((long long)d * p.ny + j) * p.psx + k0;
    prefetch_line(p.psi[FX0][AX][side] + oa);
    prefetch_line(p.psi[FX1][AX][side] + oa);
  }
  if ((HALF_H ? h_slab(j, p.jb, p.je, P, d, side) : e_slab(j, p.jb, p.je, P, d, side)) >= 0) {
    const long long oa = ((long long)i * P + d) * p.psy + k0;
    prefetch_line(p.psi[FY0][AY][side] + oa);
    prefetch_line(p.psi[FY1][AY][side] + oa);
  }
  if (zslab) {  // the side whose slab cells the group holds (the low one if both)
    const bool lo = k0 <= p.kb + P - 1 && k0 + 3 >= p.kb, hi = k0 + 3 >= p.ke - P && k0 <= p.ke - 1;
    if (lo || hi) {
      const int sd = lo ? LO : HI;
      const long long oz = ((long long)i * p.ny + j) * p.psz + (k0 - (sd ? p.ke - P : p.kb));
      prefetch_line(p.psi[FZ0][AZ][sd] + oz);
      prefetch_line(p.psi[FZ1][AZ][sd] + oz);
    }
  }
}

// Split of a row between the roles (computed on the host per job).
struct VecGeom {
  int kz0, kz1;  // vector role: k in [kz0, kz1), multiples of 4
  int nvc;       // four-cell groups per row in the vector role
  int nedge;     // edge-role cells per row: [0, kz0) and [kz1, nzp)
  int nb_vec;    // blocks of the vector role per plane (the edge role follows)
};

// One cell within one cell of the source box (widened below in i and k: the
// E CPML of Ex and Ez reads the Hy source at k + 1 and i + 1).
template <typename T> __device__ __forceinline__ bool near_src(const Params<T> &p, int i, int j, int k0, int nk) {
  return p.src_field >= 0 && i >= p.slo[0] - 1 && i < p.shi[0] && j >= p.slo[1] && j < p.shi[1] &&
         k0 + nk > p.slo[2] - 1 && k0 < p.shi[2];
}

// Edge role: four-cell groups k0 in [0, kz0) and [kz1, nzp) -- the z slabs,
// the rim and the row padding -- with the update range of every component
// tested per cell.  A group's z-slab psi values are one 16-byte vector of the
// padded z-slab rows, unless the group holds cells of both z slabs (then cell
// by cell); all old values of a group are read before the first write.
// Groups within one cell of the source box run y3_e_cell / y3_h_cell per cell.
template <typename T>
__device__ __forceinline__ bool edge_group(const Params<T> &p, const VecGeom &g, int bx, int &j, int &k0) {
  const int nge = g.nedge >> 2;
  const int t = (bx - g.nb_vec) * kVecThreads + threadIdx.x;
  if (t >= (p.je - p.jb) * nge) return false;
  const int r = t / nge, e4 = 4 * (t - r * nge);
  j = p.jb + r;
  k0 = e4 < g.kz0 ? e4 : g.kz1 + (e4 - g.kz0);
  return true;
}

template <typename T, bool EXACT>
__device__ __forceinline__ void v3_edge_e(const Params<T> &p, const VecGeom &g, int i, int bx, int s) {
  int j, k0;
  if (!edge_group(p, g, bx, j, k0)) return;
  if (near_src(p, i, j, k0, 4)) {
    for (int m = 0; m < 4; ++m)
      if (k0 + m < p.nz) y3_e_cell<T, EXACT>(p, i, j, k0 + m, p.state[0] + s, s);
    return;
  }
  using A = Ar<T, EXACT>;
  const int P = p.P;
  const bool iex = i > p.ib, jey = j > p.jb;
  bool mex[4], mey[4], mez[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int k = k0 + m;
    const bool kc = k >= p.kb && k < p.ke;
    mex[m] = iex && kc;
    mey[m] = jey && kc;
    mez[m] = k > p.kb && k < p.ke;
  }
  const int sy = p.nzp;
  const long long sx = (long long)p.ny * p.nzp, bi = (long long)i * sx;
  const int o = j * sy + k0;
  psi_prefetch<T, false>(p, i, j, k0, true);
  const T *const hx = p.f[HX] + bi, *const hy = p.f[HY] + bi, *const hz = p.f[HZ] + bi;
  V4<T> Hx, Hy, Hz, Hzy, Hxy, Hzx, Hyx, C0, C1, C2, Ex, Ey, Ez, Rz, Kz;
  ld4(Hx, hx + o);
  ld4(Hy, hy + o);
  ld4(Hz, hz + o);
  ld4(Hzy, hz + (o + sy));
  ld4(Hxy, hx + (o + sy));
  ld4(Hzx, hz + sx + o);
  ld4(Hyx, hy + sx + o);
  const bool kn = k0 + 4 < p.nzp;  // the k + 1 neighbour of the last cell
  const T hyk = kn ? __ldg(hy + (o + 4)) : T(0), hxk = kn ? __ldg(hx + (o + 4)) : T(0);
  load_cb(p, bi, o, C0, C1, C2);
  T *const ex = p.f[EX] + bi, *const ey = p.f[EY] + bi, *const ez = p.f[EZ] + bi;
  ldw4(Ex, ex + o);
  ldw4(Ey, ey + o);
  ldw4(Ez, ez + o);
  ld4(Rz, p.rkd[2] + k0);
  if (EXACT) ld4(Kz, p.kd[2] + k0);
  const T rkx = p.rkd[0][i], rky = p.rkd[1][j];
  const T kx = EXACT ? p.kd[0][i] : T(0), ky = EXACT ? p.kd[1][j] : T(0);
  T e0[4], e1[4], e2[4], dzy[4], dyz[4], dxz[4], dzx[4], dyx[4], dxy[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const T hy1 = m < 3 ? Hy.v[m + 1] : hyk, hx1 = m < 3 ? Hx.v[m + 1] : hxk;
    const T kz = EXACT ? Kz.v[m] : T(0);
    dzy[m] = A::sub(Hzy.v[m], Hz.v[m]);
    dyz[m] = A::sub(hy1, Hy.v[m]);
    dxz[m] = A::sub(hx1, Hx.v[m]);
    dzx[m] = A::sub(Hzx.v[m], Hz.v[m]);
    dyx[m] = A::sub(Hyx.v[m], Hy.v[m]);
    dxy[m] = A::sub(Hxy.v[m], Hx.v[m]);
    e0[m] = A::add(Ex.v[m], A::mul(C0.v[m], A::sub(A::div(dzy[m], ky, rky), A::div(dyz[m], kz, Rz.v[m]))));
    e1[m] = A::add(Ey.v[m], A::mul(C1.v[m], A::sub(A::div(dxz[m], kz, Rz.v[m]), A::div(dzx[m], kx, rkx))));
    e2[m] = A::add(Ez.v[m], A::mul(C2.v[m], A::sub(A::div(dyx[m], kx, rkx), A::div(dxy[m], ky, rky))));
  }
  int d, side, q;
  if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_ey_xinc, update_pml_ez_xinc
    const long long oa = ((long long)d * p.ny + j) * p.psx + k0;
    const T be = p.be[q], ce = p.ce[q];
    T *const py = p.psi[EY][AX][side] + oa, *const pz = p.psi[EZ][AX][side] + oa;
    V4<T> Py, Pz;
    ldw4(Py, py);
    ldw4(Pz, pz);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (mey[m]) {
        Py.v[m] = A::add(A::mul(be, Py.v[m]), A::div(A::mul(ce, dzx[m]), p.dx, p.rdx));
        e1[m] = A::sub(e1[m], A::mul(C1.v[m], Py.v[m]));
      }
      if (mez[m]) {
        Pz.v[m] = A::add(A::mul(be, Pz.v[m]), A::div(A::mul(ce, dyx[m]), p.dx, p.rdx));
        e2[m] = A::add(e2[m], A::mul(C2.v[m], Pz.v[m]));
      }
    }
    st4(py, Py.v);
    st4(pz, Pz.v);
  }
  if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_ex_yinc, update_pml_ez_yinc
    const long long oa = ((long long)i * P + d) * p.psy + k0;
    const T be = p.be[q], ce = p.ce[q];
    T *const px = p.psi[EX][AY][side] + oa, *const pz = p.psi[EZ][AY][side] + oa;
    V4<T> Px, Pz;
    ldw4(Px, px);
    ldw4(Pz, pz);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (mex[m]) {
        Px.v[m] = A::add(A::mul(be, Px.v[m]), A::div(A::mul(ce, dzy[m]), p.dx, p.rdx));
        e0[m] = A::add(e0[m], A::mul(C0.v[m], Px.v[m]));
      }
      if (mez[m]) {
        Pz.v[m] = A::add(A::mul(be, Pz.v[m]), A::div(A::mul(ce, dxy[m]), p.dx, p.rdx));
        e2[m] = A::sub(e2[m], A::mul(C2.v[m], Pz.v[m]));
      }
    }
    st4(px, Px.v);
    st4(pz, Pz.v);
  }
  // update_pml_ex_zinc, update_pml_ey_zinc.  The z-slab psi rows are padded to whole four-cell
  // groups: when the group's slab cells lie on one side (always unless
  // ke - kb < 2P + 3), its four values are one 16-byte aligned vector of the
  // row (the rim cells' elements are padding, written back as read);
  // otherwise cell by cell.
  int qz[4], dz[4], zside = -1;
  bool zmix = false;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    int sd = 0;
    dz[m] = 0;
    qz[m] = mex[m] || mey[m] ? e_slab(k0 + m, p.kb, p.ke, P, dz[m], sd) : -1;
    if (qz[m] >= 0) {
      zmix |= zside >= 0 && zside != sd;
      zside = sd;
    }
  }
  const long long ob = ((long long)i * p.ny + j) * p.psz;  // z-slab psi row (i, j)
  if (zside >= 0 && !zmix) {
    const int off = k0 - (zside ? p.ke - P : p.kb);  // slab index d of the group's first cell
    T *const qx = p.psi[EX][AZ][zside] + (ob + off), *const qy = p.psi[EY][AZ][zside] + (ob + off);
    V4<T> Zx, Zy;
    ldw4(Zx, qx);
    ldw4(Zy, qy);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (qz[m] < 0) continue;
      const T be = p.be[qz[m]], ce = p.ce[qz[m]];
      if (mex[m]) {
        Zx.v[m] = A::add(A::mul(be, Zx.v[m]), A::div(A::mul(ce, dyz[m]), p.dx, p.rdx));
        e0[m] = A::sub(e0[m], A::mul(C0.v[m], Zx.v[m]));
      }
      if (mey[m]) {
        Zy.v[m] = A::add(A::mul(be, Zy.v[m]), A::div(A::mul(ce, dxz[m]), p.dx, p.rdx));
        e1[m] = A::add(e1[m], A::mul(C1.v[m], Zy.v[m]));
      }
    }
    st4(qx, Zx.v);
    st4(qy, Zy.v);
  } else if (zmix) {
    T zx[4], zy[4];
    int sz[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      int dd = 0;
      sz[m] = 0;
      if (qz[m] >= 0) {e_slab(k0 + m, p.kb, p.ke, P, dd, sz[m]);}
      zx[m] = qz[m] >= 0 && mex[m] ? p.psi[EX][AZ][sz[m]][ob + dz[m]] : T(0);
      zy[m] = qz[m] >= 0 && mey[m] ? p.psi[EY][AZ][sz[m]][ob + dz[m]] : T(0);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (qz[m] < 0) continue;
      const T be = p.be[qz[m]], ce = p.ce[qz[m]];
      if (mex[m]) {
        zx[m] = A::add(A::mul(be, zx[m]), A::div(A::mul(ce, dyz[m]), p.dx, p.rdx));
        p.psi[EX][AZ][sz[m]][ob + dz[m]] = zx[m];
        e0[m] = A::sub(e0[m], A::mul(C0.v[m], zx[m]));
      }
      if (mey[m]) {
        zy[m] = A::add(A::mul(be, zy[m]), A::div(A::mul(ce, dxz[m]), p.dx, p.rdx));
        p.psi[EY][AZ][sz[m]][ob + dz[m]] = zy[m];
        e1[m] = A::add(e1[m], A::mul(C1.v[m], zy[m]));
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; ++m) {  // cells outside a component's range keep their value
    e0[m] = mex[m] ? e0[m] : Ex.v[m];
    e1[m] = mey[m] ? e1[m] : Ey.v[m];
    e2[m] = mez[m] ? e2[m] : Ez.v[m];
  }
  st4(ex + o, e0);
  st4(ey + o, e1);
  st4(ez + o, e2);
#pragma unroll
  for (int pq = 0; pq < 2; ++pq) {
    const int dm = p.port_pos[pq] - k0;
    if ((unsigned)dm < 4u) {
      const long long pc = (long long)i * p.ny + j;
#pragma unroll
      for (int m = 0; m < 4; ++m)
        if (m == dm) {
          if (mex[m]) capture(p, s, pq, 0, pc, e0[m]);
          if (mey[m]) capture(p, s, pq, 1, pc, e1[m]);
        }
    }
  }
}

template <typename T, bool EXACT, bool CG>
__device__ __forceinline__ void v3_edge_h(const Params<T> &p, const VecGeom &g, int i, int bx, int s) {
  int j, k0;
  if (!edge_group(p, g, bx, j, k0)) return;
  if (near_src(p, i, j, k0, 4)) {
    for (int m = 0; m < 4; ++m)
      if (k0 + m < p.nz) y3_h_cell<T, EXACT, CG>(p, i, j, k0 + m, p.state[0] + s, s);
    return;
  }
  using A = Ar<T, EXACT>;
  const int P = p.P;
  const bool ihy = i > p.ib, jhx = j > p.jb;
  bool mhx[4], mhy[4], mhz[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int k = k0 + m;
    const bool kc = k >= p.kb && k < p.ke, ko = k > p.kb && k < p.ke;
    mhx[m] = jhx && ko;
    mhy[m] = ihy && ko;
    mhz[m] = ihy && jhx && kc;
  }
  const int sy = p.nzp;
  const long long sx = (long long)p.ny * p.nzp, bi = (long long)i * sx;
  const int o = j * sy + k0;
  psi_prefetch<T, true>(p, i, j, k0, true);
  const T *const ex = p.f[EX] + bi, *const ey = p.f[EY] + bi, *const ez = p.f[EZ] + bi;
  V4<T> Ex, Ey, Ez, Ezy, Exy, Ezx, Eyx, Hx, Hy, Hz, Rz, Kz;
  ld4e<CG>(Ex, ex + o);
  ld4e<CG>(Ey, ey + o);
  ld4e<CG>(Ez, ez + o);
  ld4e<CG>(Ezy, ez + (o - sy));
  ld4e<CG>(Exy, ex + (o - sy));
  ld4e<CG>(Ezx, ez - sx + o);
  ld4e<CG>(Eyx, ey - sx + o);
  const bool kp = k0 > 0;  // the k - 1 neighbour of the first cell
  const T eyk = kp ? ld_e<CG>(ey + (o - 1)) : T(0), exk = kp ? ld_e<CG>(ex + (o - 1)) : T(0);
  T *const hx = p.f[HX] + bi, *const hy = p.f[HY] + bi, *const hz = p.f[HZ] + bi;
  ldw4(Hx, hx + o);
  ldw4(Hy, hy + o);
  ldw4(Hz, hz + o);
  ld4(Rz, p.rkd[5] + k0);
  if (EXACT) ld4(Kz, p.kd[5] + k0);
  const T rkx = p.rkd[3][i], rky = p.rkd[4][j];
  const T kx = EXACT ? p.kd[3][i] : T(0), ky = EXACT ? p.kd[4][j] : T(0);
  const T db = p.db;
  T h0[4], h1[4], h2[4], dyz[4], dzy[4], dzx[4], dxz[4], dxy[4], dyx[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const T ey1 = m > 0 ? Ey.v[m - 1] : eyk, ex1 = m > 0 ? Ex.v[m - 1] : exk;
    const T kz = EXACT ? Kz.v[m] : T(0);
    dyz[m] = A::sub(Ey.v[m], ey1);
    dzy[m] = A::sub(Ez.v[m], Ezy.v[m]);
    dzx[m] = A::sub(Ez.v[m], Ezx.v[m]);
    dxz[m] = A::sub(Ex.v[m], ex1);
    dxy[m] = A::sub(Ex.v[m], Exy.v[m]);
    dyx[m] = A::sub(Ey.v[m], Eyx.v[m]);
    h0[m] = A::add(Hx.v[m], A::mul(db, A::sub(A::div(dyz[m], kz, Rz.v[m]), A::div(dzy[m], ky, rky))));
    h1[m] = A::add(Hy.v[m], A::mul(db, A::sub(A::div(dzx[m], kx, rkx), A::div(dxz[m], kz, Rz.v[m]))));
    h2[m] = A::add(Hz.v[m], A::mul(db, A::sub(A::div(dxy[m], ky, rky), A::div(dyx[m], kx, rkx))));
  }
  int d, side, q;
  if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_hy_xinc, update_pml_hz_xinc
    const long long oa = ((long long)d * p.ny + j) * p.psx + k0;
    const T bh = p.bh[q], ch = p.ch[q];
    T *const py = p.psi[HY][AX][side] + oa, *const pz = p.psi[HZ][AX][side] + oa;
    V4<T> Py, Pz;
    ldw4(Py, py);
    ldw4(Pz, pz);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (mhy[m]) {
        Py.v[m] = A::add(A::mul(bh, Py.v[m]), A::div(A::mul(ch, dzx[m]), p.dx, p.rdx));
        h1[m] = A::add(h1[m], A::mul(db, Py.v[m]));
      }
      if (mhz[m]) {
        Pz.v[m] = A::add(A::mul(bh, Pz.v[m]), A::div(A::mul(ch, dyx[m]), p.dx, p.rdx));
        h2[m] = A::sub(h2[m], A::mul(db, Pz.v[m]));
      }
    }
    st4(py, Py.v);
    st4(pz, Pz.v);
  }
  if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_hx_yinc, update_pml_hz_yinc
    const long long oa = ((long long)i * P + d) * p.psy + k0;
    const T bh = p.bh[q], ch = p.ch[q];
    T *const px = p.psi[HX][AY][side] + oa, *const pz = p.psi[HZ][AY][side] + oa;
    V4<T> Px, Pz;
    ldw4(Px, px);
    ldw4(Pz, pz);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (mhx[m]) {
        Px.v[m] = A::add(A::mul(bh, Px.v[m]), A::div(A::mul(ch, dzy[m]), p.dx, p.rdx));
        h0[m] = A::sub(h0[m], A::mul(db, Px.v[m]));
      }
      if (mhz[m]) {
        Pz.v[m] = A::add(A::mul(bh, Pz.v[m]), A::div(A::mul(ch, dxy[m]), p.dx, p.rdx));
        h2[m] = A::add(h2[m], A::mul(db, Pz.v[m]));
      }
    }
    st4(px, Px.v);
    st4(pz, Pz.v);
  }
  // update_pml_hx_zinc, update_pml_hy_zinc.  The z-slab psi rows are padded to whole four-cell
  // groups: when the group's slab cells lie on one side (always unless
  // ke - kb < 2P + 3), its four values are one 16-byte aligned vector of the
  // row (the rim cells' elements are padding, written back as read);
  // otherwise cell by cell.
  int qz[4], dz[4], zside = -1;
  bool zmix = false;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    int sd = 0;
    dz[m] = 0;
    qz[m] = mhx[m] || mhy[m] ? h_slab(k0 + m, p.kb, p.ke, P, dz[m], sd) : -1;
    if (qz[m] >= 0) {
      zmix |= zside >= 0 && zside != sd;
      zside = sd;
    }
  }
  const long long ob = ((long long)i * p.ny + j) * p.psz;  // z-slab psi row (i, j)
  if (zside >= 0 && !zmix) {
    const int off = k0 - (zside ? p.ke - P : p.kb);  // slab index d of the group's first cell
    T *const qx = p.psi[HX][AZ][zside] + (ob + off), *const qy = p.psi[HY][AZ][zside] + (ob + off);
    V4<T> Zx, Zy;
    ldw4(Zx, qx);
    ldw4(Zy, qy);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (qz[m] < 0) continue;
      const T bh = p.bh[qz[m]], ch = p.ch[qz[m]];
      if (mhx[m]) {
        Zx.v[m] = A::add(A::mul(bh, Zx.v[m]), A::div(A::mul(ch, dyz[m]), p.dx, p.rdx));
        h0[m] = A::add(h0[m], A::mul(db, Zx.v[m]));
      }
      if (mhy[m]) {
        Zy.v[m] = A::add(A::mul(bh, Zy.v[m]), A::div(A::mul(ch, dxz[m]), p.dx, p.rdx));
        h1[m] = A::sub(h1[m], A::mul(db, Zy.v[m]));
      }
    }
    st4(qx, Zx.v);
    st4(qy, Zy.v);
  } else if (zmix) {
    T zx[4], zy[4];
    int sz[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      int dd = 0;
      sz[m] = 0;
      if (qz[m] >= 0) {h_slab(k0 + m, p.kb, p.ke, P, dd, sz[m]);}
      zx[m] = qz[m] >= 0 && mhx[m] ? p.psi[HX][AZ][sz[m]][ob + dz[m]] : T(0);
      zy[m] = qz[m] >= 0 && mhy[m] ? p.psi[HY][AZ][sz[m]][ob + dz[m]] : T(0);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (qz[m] < 0) continue;
      const T bh = p.bh[qz[m]], ch = p.ch[qz[m]];
      if (mhx[m]) {
        zx[m] = A::add(A::mul(bh, zx[m]), A::div(A::mul(ch, dyz[m]), p.dx, p.rdx));
        p.psi[HX][AZ][sz[m]][ob + dz[m]] = zx[m];
        h0[m] = A::add(h0[m], A::mul(db, zx[m]));
      }
      if (mhy[m]) {
        zy[m] = A::add(A::mul(bh, zy[m]), A::div(A::mul(ch, dxz[m]), p.dx, p.rdx));
        p.psi[HY][AZ][sz[m]][ob + dz[m]] = zy[m];
        h1[m] = A::sub(h1[m], A::mul(db, zy[m]));
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    h0[m] = mhx[m] ? h0[m] : Hx.v[m];
    h1[m] = mhy[m] ? h1[m] : Hy.v[m];
    h2[m] = mhz[m] ? h2[m] : Hz.v[m];
  }
  st4(hx + o, h0);
  st4(hy + o, h1);
  st4(hz + o, h2);
#pragma unroll
  for (int pq = 0; pq < 2; ++pq) {
    const int dm = p.port_pos[pq] - k0;
    if ((unsigned)(dm + 1) < 5u) {
      const long long pc = (long long)i * p.ny + j;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (m == dm) {
          if (mhx[m]) capture(p, s, pq, 2, pc, h0[m]);
          if (mhy[m]) capture(p, s, pq, 4, pc, h1[m]);
        }
        if (m == dm + 1) {
          if (mhx[m]) capture(p, s, pq, 3, pc, h0[m]);
          if (mhy[m]) capture(p, s, pq, 5, pc, h1[m]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// E half-step.  Updated: Ex i (ib,ie) j [jb,je) k [kb,ke); Ey i [ib,ie)
// j (jb,je) k [kb,ke); Ez i [ib,ie) j [jb,je) k (kb,ke).  Grid: (vector-role
// then edge-role blocks, x-planes ib..ie-1).
// ---------------------------------------------------------------------------
// One block of x-plane i: bx < nb_vec a vector-role block, the edge role above.
template <typename T, bool EXACT>
__device__ __forceinline__ void v3_e_block(const Params<T> &p, const VecGeom &g, int i, int bx, int s) {
  if (bx >= g.nb_vec) {
    v3_edge_e<T, EXACT>(p, g, i, bx, s);
    return;
  }
  const int t = bx * kVecThreads + threadIdx.x;
  if (t >= (p.je - p.jb) * g.nvc) return;
  const int r = t / g.nvc;
  const int j = p.jb + r, k0 = g.kz0 + 4 * (t - r * g.nvc);
  if (near_src(p, i, j, k0, 4) && p.src_field == HY) {
    for (int m = 0; m < 4; ++m) y3_e_cell<T, EXACT>(p, i, j, k0 + m, p.state[0] + s, s);
    return;
  }
  using A = Ar<T, EXACT>;
  const int sy = p.nzp;
  const long long sx = (long long)p.ny * p.nzp, bi = (long long)i * sx;
  const int o = j * sy + k0;
  const T *const hx = p.f[HX] + bi, *const hy = p.f[HY] + bi, *const hz = p.f[HZ] + bi;
  V4<T> Hx, Hy, Hz, Hzy, Hxy, Hzx, Hyx, C0, C1, C2, Ex, Ey, Ez, Rz, Kz;
  ld4(Hx, hx + o);
  ld4(Hy, hy + o);
  ld4(Hz, hz + o);
  ld4(Hzy, hz + (o + sy));
  ld4(Hxy, hx + (o + sy));
  ld4(Hzx, hz + sx + o);
  ld4(Hyx, hy + sx + o);
  const T hyk = __ldg(hy + (o + 4)), hxk = __ldg(hx + (o + 4));  // k0 + 4 < kz1 <= nz - 2
  load_cb(p, bi, o, C0, C1, C2);
  T *const ex = p.f[EX] + bi, *const ey = p.f[EY] + bi, *const ez = p.f[EZ] + bi;
  ldw4(Ex, ex + o);
  ldw4(Ey, ey + o);
  ldw4(Ez, ez + o);
  ld4(Rz, p.rkd[2] + k0);
  if (EXACT) ld4(Kz, p.kd[2] + k0);
  const T rkx = p.rkd[0][i], rky = p.rkd[1][j];
  const T kx = EXACT ? p.kd[0][i] : T(0), ky = EXACT ? p.kd[1][j] : T(0);
  // update ranges: all four cells are inside (kb, ke); Ex leaves out i = ib,
  // Ey j = jb
  const bool mex = i > p.ib, mey = j > p.jb;
  T e0[4], e1[4], e2[4], dzy[4], dyz[4], dxz[4], dzx[4], dyx[4], dxy[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const T hy1 = m < 3 ? Hy.v[m + 1] : hyk, hx1 = m < 3 ? Hx.v[m + 1] : hxk;
    const T kz = EXACT ? Kz.v[m] : T(0);
    dzy[m] = A::sub(Hzy.v[m], Hz.v[m]);
    dyz[m] = A::sub(hy1, Hy.v[m]);
    dxz[m] = A::sub(hx1, Hx.v[m]);
    dzx[m] = A::sub(Hzx.v[m], Hz.v[m]);
    dyx[m] = A::sub(Hyx.v[m], Hy.v[m]);
    dxy[m] = A::sub(Hxy.v[m], Hx.v[m]);
    e0[m] = A::add(Ex.v[m], A::mul(C0.v[m], A::sub(A::div(dzy[m], ky, rky), A::div(dyz[m], kz, Rz.v[m]))));
    e1[m] = A::add(Ey.v[m], A::mul(C1.v[m], A::sub(A::div(dxz[m], kz, Rz.v[m]), A::div(dzx[m], kx, rkx))));
    e2[m] = A::add(Ez.v[m], A::mul(C2.v[m], A::sub(A::div(dyx[m], kx, rkx), A::div(dxy[m], ky, rky))));
  }
  // soft source on Ey ('TE'): after the curl, before the CPML terms
  if (p.src_field == EY && mey && i >= p.slo[0] && i < p.shi[0] && j >= p.slo[1] && j < p.shi[1] &&
      k0 + 4 > p.slo[2] && k0 < p.shi[2]) {
    const T Jn = p.jsrc[p.state[0] + s];
#pragma unroll
    for (int m = 0; m < 4; ++m)
      if (k0 + m >= p.slo[2] && k0 + m < p.shi[2]) e1[m] = A::sub(e1[m], Jn);
  }
  const int P = p.P;
  int d, side, q;
  if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_ey_xinc, update_pml_ez_xinc
    const long long oa = ((long long)d * p.ny + j) * p.psx + k0;
    const T be = p.be[q], ce = p.ce[q];
    if (mey) {
      T *const py = p.psi[EY][AX][side] + oa;
      V4<T> Py;
      ldw4(Py, py);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        Py.v[m] = A::add(A::mul(be, Py.v[m]), A::div(A::mul(ce, dzx[m]), p.dx, p.rdx));
        e1[m] = A::sub(e1[m], A::mul(C1.v[m], Py.v[m]));
      }
      st4(py, Py.v);
    }
    T *const pz = p.psi[EZ][AX][side] + oa;
    V4<T> Pz;
    ldw4(Pz, pz);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      Pz.v[m] = A::add(A::mul(be, Pz.v[m]), A::div(A::mul(ce, dyx[m]), p.dx, p.rdx));
      e2[m] = A::add(e2[m], A::mul(C2.v[m], Pz.v[m]));
    }
    st4(pz, Pz.v);
  }
  if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_ex_yinc, update_pml_ez_yinc
    const long long oa = ((long long)i * P + d) * p.psy + k0;
    const T be = p.be[q], ce = p.ce[q];
    if (mex) {
      T *const px = p.psi[EX][AY][side] + oa;
      V4<T> Px;
      ldw4(Px, px);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        Px.v[m] = A::add(A::mul(be, Px.v[m]), A::div(A::mul(ce, dzy[m]), p.dx, p.rdx));
        e0[m] = A::add(e0[m], A::mul(C0.v[m], Px.v[m]));
      }
      st4(px, Px.v);
    }
    T *const pz = p.psi[EZ][AY][side] + oa;
    V4<T> Pz;
    ldw4(Pz, pz);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      Pz.v[m] = A::add(A::mul(be, Pz.v[m]), A::div(A::mul(ce, dxy[m]), p.dx, p.rdx));
      e2[m] = A::sub(e2[m], A::mul(C2.v[m], Pz.v[m]));
    }
    st4(pz, Pz.v);
  }
  if (mex) st4(ex + o, e0);
  if (mey) st4(ey + o, e1);
  st4(ez + o, e2);
  // port planes: raw Ex, Ey samples for the DFT fold
#pragma unroll
  for (int pq = 0; pq < 2; ++pq) {
    const int dm = p.port_pos[pq] - k0;
    if ((unsigned)dm < 4u) {
      const long long pc = (long long)i * p.ny + j;
#pragma unroll
      for (int m = 0; m < 4; ++m)
        if (m == dm) {
          if (mex) capture(p, s, pq, 0, pc, e0[m]);
          if (mey) capture(p, s, pq, 1, pc, e1[m]);
        }
    }
  }
}

// ---------------------------------------------------------------------------
// H half-step.  Updated: Hx i [ib,ie) j (jb,je) k (kb,ke); Hy i (ib,ie)
// j [jb,je) k (kb,ke); Hz i (ib,ie) j (jb,je) k [kb,ke).  Planes run in
// decreasing i: the launch starts on the E planes the E half-step wrote last
// (still in L2) and ends on the planes the next E half-step reads first.
// ---------------------------------------------------------------------------
template <typename T, bool EXACT, bool CG>
__device__ __forceinline__ void v3_h_block(const Params<T> &p, const VecGeom &g, int i, int bx, int s) {
  if (bx >= g.nb_vec) {
    v3_edge_h<T, EXACT, CG>(p, g, i, bx, s);
    return;
  }
  const int t = bx * kVecThreads + threadIdx.x;
  if (t >= (p.je - p.jb) * g.nvc) return;
  const int r = t / g.nvc;
  const int j = p.jb + r, k0 = g.kz0 + 4 * (t - r * g.nvc);
  using A = Ar<T, EXACT>;
  const int sy = p.nzp;
  const long long sx = (long long)p.ny * p.nzp, bi = (long long)i * sx;
  const int o = j * sy + k0;
  psi_prefetch<T, true>(p, i, j, k0, false);
  const T *const ex = p.f[EX] + bi, *const ey = p.f[EY] + bi, *const ez = p.f[EZ] + bi;
  V4<T> Ex, Ey, Ez, Ezy, Exy, Ezx, Eyx, Hx, Hy, Hz, Rz, Kz;
  ld4e<CG>(Ex, ex + o);
  ld4e<CG>(Ey, ey + o);
  ld4e<CG>(Ez, ez + o);
  ld4e<CG>(Ezy, ez + (o - sy));
  ld4e<CG>(Exy, ex + (o - sy));
  ld4e<CG>(Ezx, ez - sx + o);
  ld4e<CG>(Eyx, ey - sx + o);
  const T eyk = ld_e<CG>(ey + (o - 1)), exk = ld_e<CG>(ex + (o - 1));  // k0 - 1 >= kz0 - 1 >= kb + P - 1
  T *const hx = p.f[HX] + bi, *const hy = p.f[HY] + bi, *const hz = p.f[HZ] + bi;
  ldw4(Hx, hx + o);
  ldw4(Hy, hy + o);
  ldw4(Hz, hz + o);
  ld4(Rz, p.rkd[5] + k0);
  if (EXACT) ld4(Kz, p.kd[5] + k0);
  const T rkx = p.rkd[3][i], rky = p.rkd[4][j];
  const T kx = EXACT ? p.kd[3][i] : T(0), ky = EXACT ? p.kd[4][j] : T(0);
  const T db = p.db;
  // update ranges: all four cells are inside (kb, ke); Hx leaves out j = jb,
  // Hy i = ib, Hz both
  const bool mhx = j > p.jb, mhy = i > p.ib, mhz = mhx && mhy;
  // soft source on Hy ('TM'): subtracted before the Hy update
  const bool src = p.src_field == HY && mhy && i >= p.slo[0] && i < p.shi[0] && j >= p.slo[1] && j < p.shi[1] &&
                   k0 + 4 > p.slo[2] && k0 < p.shi[2];
  const T Jn = src ? p.jsrc[p.state[0] + s] : T(0);
  T h0[4], h1[4], h2[4], dyz[4], dzy[4], dzx[4], dxz[4], dxy[4], dyx[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const T ey1 = m > 0 ? Ey.v[m - 1] : eyk, ex1 = m > 0 ? Ex.v[m - 1] : exk;
    const T kz = EXACT ? Kz.v[m] : T(0);
    dyz[m] = A::sub(Ey.v[m], ey1);
    dzy[m] = A::sub(Ez.v[m], Ezy.v[m]);
    dzx[m] = A::sub(Ez.v[m], Ezx.v[m]);
    dxz[m] = A::sub(Ex.v[m], ex1);
    dxy[m] = A::sub(Ex.v[m], Exy.v[m]);
    dyx[m] = A::sub(Ey.v[m], Eyx.v[m]);
    T hy0 = Hy.v[m];
    if (src && k0 + m >= p.slo[2] && k0 + m < p.shi[2]) hy0 = A::sub(hy0, Jn);
    h0[m] = A::add(Hx.v[m], A::mul(db, A::sub(A::div(dyz[m], kz, Rz.v[m]), A::div(dzy[m], ky, rky))));
    h1[m] = A::add(hy0, A::mul(db, A::sub(A::div(dzx[m], kx, rkx), A::div(dxz[m], kz, Rz.v[m]))));
    h2[m] = A::add(Hz.v[m], A::mul(db, A::sub(A::div(dxy[m], ky, rky), A::div(dyx[m], kx, rkx))));
  }
  const int P = p.P;
  int d, side, q;
  if (mhy && (q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_hy_xinc, update_pml_hz_xinc
    const long long oa = ((long long)d * p.ny + j) * p.psx + k0;
    const T bh = p.bh[q], ch = p.ch[q];
    T *const py = p.psi[HY][AX][side] + oa;
    V4<T> Py;
    ldw4(Py, py);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      Py.v[m] = A::add(A::mul(bh, Py.v[m]), A::div(A::mul(ch, dzx[m]), p.dx, p.rdx));
      h1[m] = A::add(h1[m], A::mul(db, Py.v[m]));
    }
    st4(py, Py.v);
    if (mhz) {
      T *const pz = p.psi[HZ][AX][side] + oa;
      V4<T> Pz;
      ldw4(Pz, pz);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        Pz.v[m] = A::add(A::mul(bh, Pz.v[m]), A::div(A::mul(ch, dyx[m]), p.dx, p.rdx));
        h2[m] = A::sub(h2[m], A::mul(db, Pz.v[m]));
      }
      st4(pz, Pz.v);
    }
  }
  if (mhx && (q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_hx_yinc, update_pml_hz_yinc
    const long long oa = ((long long)i * P + d) * p.psy + k0;
    const T bh = p.bh[q], ch = p.ch[q];
    T *const px = p.psi[HX][AY][side] + oa;
    V4<T> Px;
    ldw4(Px, px);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      Px.v[m] = A::add(A::mul(bh, Px.v[m]), A::div(A::mul(ch, dzy[m]), p.dx, p.rdx));
      h0[m] = A::sub(h0[m], A::mul(db, Px.v[m]));
    }
    st4(px, Px.v);
    if (mhz) {
      T *const pz = p.psi[HZ][AY][side] + oa;
      V4<T> Pz;
      ldw4(Pz, pz);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        Pz.v[m] = A::add(A::mul(bh, Pz.v[m]), A::div(A::mul(ch, dxy[m]), p.dx, p.rdx));
        h2[m] = A::add(h2[m], A::mul(db, Pz.v[m]));
      }
      st4(pz, Pz.v);
    }
  }
  if (mhx) st4(hx + o, h0);
  if (mhy) st4(hy + o, h1);
  if (mhz) st4(hz + o, h2);
  // port planes: raw Hx, Hy at k = port and port + 1
#pragma unroll
  for (int pq = 0; pq < 2; ++pq) {
    const int dm = p.port_pos[pq] - k0;
    if ((unsigned)(dm + 1) < 5u) {  // k = port or port + 1 among the four cells
      const long long pc = (long long)i * p.ny + j;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (m == dm) {
          if (mhx) capture(p, s, pq, 2, pc, h0[m]);
          if (mhy) capture(p, s, pq, 4, pc, h1[m]);
        }
        if (m == dm + 1) {
          if (mhx) capture(p, s, pq, 3, pc, h0[m]);
          if (mhy) capture(p, s, pq, 5, pc, h1[m]);
        }
      }
    }
  }
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kVecThreads, sizeof(T) == 4 ? kVecBlocksPerSME : 3) k_v3_e(Params<T> p, VecGeom g, int s) {
  pdl_wait();
  v3_e_block<T, EXACT>(p, g, p.ib + blockIdx.y, blockIdx.x, s);
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kVecThreads, sizeof(T) == 4 ? kVecBlocksPerSM : 3) k_v3_h(Params<T> p, VecGeom g, int s) {
  pdl_wait();
  v3_h_block<T, EXACT, false>(p, g, p.ie - 1 - blockIdx.y, blockIdx.x, s);
}

// ---------------------------------------------------------------------------
// Ordered form: one launch per time step runs both half-steps, plane by
// plane: E(0) .. E(D-1), then for q = 0 .. n-1 the pair E(q+D) (while q+D <
// n), H(q) -- a unit of nb blocks each, n = ie - ib updated planes, q = i -
// ib, D the lag (wave.lag).  H(q) reads new E of planes q and q-1 and
// overwrites the H of plane q that E(q) and E(q-1) read, so its blocks wait
// until every block of E(q) and E(q-1) has finished; no other dependence
// exists inside a step.  A block's place in the order is its block index; the
// hardware dispatches a 1D grid in increasing block index, so the E blocks an
// H block waits for were dispatched D units or more earlier, and those never
// wait: the waits end, and with the lag they are rarely needed at all.  Each
// wait is bounded (kWaitCycles); on expiry the block records state[1] = 2
// and returns without updating, and oidt_job_sync reports the job as timed
// out -- should a dependence ever not be resident, the launch ends with that
// error instead of hanging.  H blocks read E through L2 (another SM's L1 may
// hold lines written in this launch).  The new E of planes q and q-1 and the
// H of plane q were touched D units earlier, and D is chosen so that D planes
// of the step's arrays fit in L2: H reads them from L2 and DRAM carries each
// field word about once per step.
// ---------------------------------------------------------------------------
struct WaveArgs {
  int *done;  // [n]: E blocks finished per plane, summed over the steps run
  int nb;     // blocks per plane and half-step (vector + edge role)
  int lag;    // D, 1 <= D <= n
};

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kVecThreads, sizeof(T) == 4 ? kVecBlocksPerSM : 3)
    k_v3_wave(Params<T> p, VecGeom g, WaveArgs w, int s) {
  pdl_wait();
  __shared__ int s_ok;
  const int n = p.ie - p.ib, D = w.lag;
  const int u = (int)(blockIdx.x / w.nb), bx = (int)(blockIdx.x - (unsigned)u * w.nb);
  bool is_h;
  int q;
  if (u < D) {
    is_h = false;
    q = u;
  } else if (u < D + 2 * (n - D)) {
    const int r = u - D;
    is_h = r & 1;
    q = is_h ? r >> 1 : (r >> 1) + D;
  } else {
    is_h = true;
    q = n - D + (u - D - 2 * (n - D));
  }
  if (!is_h) {
    v3_e_block<T, EXACT>(p, g, p.ib + q, bx, s);
    __threadfence();  // this thread's stores visible to the whole GPU ...
    __syncthreads();  // ... for every thread of the block, before the count
    if (threadIdx.x == 0) atomicAdd(w.done + q, 1);
    return;
  }
  if (threadIdx.x == 0) {
    s_ok = 1;
    const int want = (int)(((long long)p.state[0] + s + 1) * w.nb);  // counts after this step's E
    const long long t0 = clock64();
    for (int d = 0; d < 2 && q - d >= 0 && s_ok; ++d)
      while (ld_acquire(w.done + (q - d)) < want)
        if (clock64() - t0 > kWaitCycles) {
          atomicExch(p.state + 1, 2);  // reported to the host by oidt_job_sync
          s_ok = 0;
          break;
        }
  }
  __syncthreads();
  if (s_ok) v3_h_block<T, EXACT, true>(p, g, p.ib + q, bx, s);
}

}  // namespace oidt
