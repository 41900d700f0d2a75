// kernels.cuh -- per-cell Yee updates for the three reference solvers, with
// the CPML psi recursion, the soft source and the port-plane capture fused in.
//
// One thread owns one cell and applies, for each field component it updates,
// exactly the sequence of operations the reference applies to that cell in
// one time step: curl update, source, then the CPML corrections in the
// reference's launch order.  With Ar<T, true> (OIDT_ARITH_EXACT) every
// operation is an IEEE add/sub/mul/div in the reference's operand order, so
// float64 results equal the reference's float64 results bit for bit.
//
// Reference kernels restated here:
//   TM2  FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_funcs.py:43-124
//   TE2  FDTD/GPU/FDTD_2D_TE/s-parameter_extraction/fdtd_funcs.py:43-124
//   3D   FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_funcs.py:43-266
// and the per-step launch order of fdtd_main.py:275-304 (3D :357-406).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace oidt {

enum { EX = 0, EY = 1, EZ = 2, HX = 3, HY = 4, HZ = 5 };
enum { AX = 0, AY = 1, AZ = 2 };
enum { LO = 0, HI = 1 };

// ---------------------------------------------------------------------------
// Arithmetic policy.
// ---------------------------------------------------------------------------
// EXACT division a / b rounded to nearest, from y = RN(1/b) (the correctly
// rounded reciprocal, computed on the host in the same precision) by two FMA
// corrections: q1 = RN(q0 + r0 y), q2 = RN(q1 + r1 y) with q0 = RN(a y) and
// the exact residuals r = a - b q.  q1 is within one ulp of a / b, so q2 is
// the correctly rounded quotient by Markstein's theorem (P. Markstein, IBM J.
// Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point
// Arithmetic, the division chapter), provided nothing under- or overflows:
// the numerator, the quotient and the reciprocal stay within [2^-lo, 2^lo]
// (the residuals are then exact); outside that range, and for NaN, the
// quotient is divided directly.  Zero numerators give a zero of either sign.
template <typename T, bool EXACT> struct Ar;
template <> struct Ar<float, true> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b, float y) {
    const float q0 = __fmul_rn(a, y);
    const float aa = fabsf(a), aq = fabsf(q0), ay = fabsf(y);
    const bool ok = (a == 0.0f || (aa >= 0x1p-100f && aa <= 0x1p+100f && aq >= 0x1p-100f && aq <= 0x1p+100f)) &&
                    ay >= 0x1p-100f && ay <= 0x1p+100f;
    if (!ok) return __fdiv_rn(a, b);
    const float q1 = __fmaf_rn(__fmaf_rn(-b, q0, a), y, q0);
    return __fmaf_rn(__fmaf_rn(-b, q1, a), y, q1);
  }
};
template <> struct Ar<float, false> {
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
  static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
  static __device__ __forceinline__ float div(float a, float, float rb) { return a * rb; }
};
template <> struct Ar<double, true> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b, double y) {
    const double q0 = __dmul_rn(a, y);
    const double aa = fabs(a), aq = fabs(q0), ay = fabs(y);
    const bool ok = (a == 0.0 || (aa >= 0x1p-900 && aa <= 0x1p+900 && aq >= 0x1p-900 && aq <= 0x1p+900)) &&
                    ay >= 0x1p-900 && ay <= 0x1p+900;
    if (!ok) return __ddiv_rn(a, b);
    const double q1 = __fma_rn(__fma_rn(-b, q0, a), y, q0);
    return __fma_rn(__fma_rn(-b, q1, a), y, q1);
  }
};
template <> struct Ar<double, false> {
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
  static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
  static __device__ __forceinline__ double div(double a, double, double rb) { return a * rb; }
};

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  The kernels of a time step are launched with
// the programmatic-serialization attribute, so a kernel may start while the
// previous kernel in its stream drains; each calls pdl_wait() before its first
// global-memory access, which returns once that kernel has completed and its
// writes are visible.  Launched without the attribute, it returns at once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Bound on every in-kernel wait for other blocks' or copies' progress.
constexpr long long kWaitCycles = 4000000000LL;  // about 2 s at 1.9 GHz

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------------------
// Job parameters (device-resident copy for batched launches).
// ---------------------------------------------------------------------------
template <typename T> struct Params {
  int mode;              // OIDT_MODE_*
  int nx, ny, nz;        // nz = 1 in 2D
  int nzp;               // 3D row pitch along z (elements); 2D: 1
  int P, ib, jb, kb, ie, je, ke;
  T *f[6];               // fields (read; updated in place by the per-cell launches)
  T *fn[6];              // fields written by the plane sweep (the other buffer)
  const T *cb[3];        // dt/eps per E component (TM2 uses cb[2] for Ez)
  const unsigned char *mat;  // 3D material index [nx][ny][nzp] (nullptr: none) ...
  const T *mtab;             // ... and its table [256][4] (CBX, CBY, CBZ, 0)
  const T *kd[6];        // kappa*dx: kxe kye kze kxh kyh kzh
  const T *rkd[6];       // reciprocals
  const T *be, *ce, *bh, *ch;
  T db, dx, rdx;
  T *psi[6][3][2];       // [field][slab axis][side] (read; H psi updated in place)
  T *psin[6][3][2];      // E psi written (== psi for the per-cell launches)
  int psx, psy;          // row pitch (elements along z) of the x- and y-slab psi arrays:
                         // nz (the reference layout) or nzp (16-byte rows, vector form)
  int psz;               // row pitch of the z-slab psi arrays: P (the reference layout), or
                         // the vector form's rows of whole four-cell groups (psi[f][AZ][side]
                         // then points at slab cell d = 0 of row 0, inside the padded row)
  const void *tmap_f;    // plane sweep: 6 CUtensorMaps of f[] (device memory)
  const void *tmap_cb;   // plane sweep: 3 CUtensorMaps of cb[]
  long long wait_cycles; // plane sweep: bound on each wait for a plane's tile loads
  int src_field;         // -1: none
  int slo[3], shi[3];
  const T *jsrc;
  T *ring;               // capture ring [K][2 ports][slots][plane]
  int ring_K, nslot;
  long long plane;       // 2D: ny, 3D: nx*ny
  int port_pos[2];
  int *state;            // state[0] = absolute step of ring slot 0
};

template <typename T>
__device__ __forceinline__ bool in_src(const Params<T> &p, int fld, int i, int j, int k) {
  return p.src_field == fld && i >= p.slo[0] && i < p.shi[0] && j >= p.slo[1] && j < p.shi[1] &&
         k >= p.slo[2] && k < p.shi[2];
}

// psi array index for a 3D slab array whose `axis` extent is P: x-slabs
// [P][ny][psx], y-slabs [nx][P][psy], z-slabs [nx][ny][psz].
template <typename T>
__device__ __forceinline__ long long psi_idx3(const Params<T> &p, int axis, int i, int j, int k) {
  if (axis == AX) return ((long long)i * p.ny + j) * p.psx + k;  // i is the slab index d
  if (axis == AY) return ((long long)i * p.P + j) * p.psy + k;   // j is d
  return ((long long)i * p.ny + j) * p.psz + k;                  // k is d
}

// E-field CPML slab test along one axis: returns coefficient index or -1,
// writes slab index d and side.  Low slab cells b..b+P-1 (coef P-1-d), high
// slab cells e-P..e-1 (coef d).  (fdtd_funcs.py update_pml_e*: be[-(d+1)],
// be[d].)
__device__ __forceinline__ int e_slab(int c, int b, int e, int P, int &d, int &side) {
  if (c >= b && c < b + P) { d = c - b; side = LO; return P - 1 - d; }
  if (c >= e - P && c < e) { d = c - (e - P); side = HI; return d; }
  return -1;
}
// H-field CPML slab: low cells b+1..b+P-1 (coef P-d), high e-P+1..e-1 (coef
// d), d in 1..P-1.  (update_pml_h*: ``i > 0 and i < pmle``, bh[-d], bh[d].)
__device__ __forceinline__ int h_slab(int c, int b, int e, int P, int &d, int &side) {
  if (c > b && c < b + P) { d = c - b; side = LO; return P - d; }
  if (c > e - P && c < e) { d = c - (e - P); side = HI; return d; }
  return -1;
}

template <typename T>
__device__ __forceinline__ void capture(const Params<T> &p, int s, int port, int slot, long long idx,
                                        T v) {
  p.ring[(((long long)s * 2 + port) * p.nslot + slot) * p.plane + idx] = v;
}

// ---------------------------------------------------------------------------
// 3D Yee (FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_funcs.py)
//
// The arithmetic of one cell lives in y3_e_compute / y3_h_compute, written
// against an accessor: the per-cell launch reads neighbours from global
// memory (GlobalAcc3), the plane-sweep kernel from shared-memory tiles.  Both
// therefore perform the identical operation sequence.
// Accessor interface:
//   h(f, di, dj, dk)   old H component f at (i+di, j+dj, k+dk), di,dj,dk in {0,1}
//   e(f, di, dj, dk)   new E component f at (i+di, j+dj, k+dk), offsets in {-1,0}
//   eold(f), hold(f), cb(a)
// ---------------------------------------------------------------------------
// Loads of E in an H update: L2 only (CG) where the same launch may have
// written E on another SM (an SM's L1 is not kept coherent with those writes),
// the read-only path otherwise.
template <bool CG, typename T> __device__ __forceinline__ T ld_e(const T *q) { return CG ? __ldcg(q) : __ldg(q); }

template <typename T, bool CG = false> struct GlobalAcc3 {
  const Params<T> &p;
  long long c, sy, sx;
  __device__ __forceinline__ T h(int f, int di, int dj, int dk) const { return p.f[f][c + di * sx + dj * sy + dk]; }
  __device__ __forceinline__ T e(int f, int di, int dj, int dk) const {
    return CG ? __ldcg(p.f[f] + (c + di * sx + dj * sy + dk)) : p.f[f][c + di * sx + dj * sy + dk];
  }
  __device__ __forceinline__ T eold(int f) const { return p.f[f][c]; }
  __device__ __forceinline__ T hold(int f) const { return p.f[f][c]; }
  __device__ __forceinline__ T cb(int a) const { return p.cb[a][c]; }
};

// New E at cell (i, j, k) -> out[EX..EZ] (old value where a component is not
// updated).  own: write the new CPML psi (else only read it: halo cells of a
// sweep tile).  Returns a bit mask of the updated components.
template <typename T, bool EXACT, class Acc>
__device__ __forceinline__ int y3_e_compute(const Params<T> &p, const Acc &a, int i, int j, int k, int n, bool own,
                                            T out[3]) {
  using A = Ar<T, EXACT>;
  const int P = p.P;
  const T Jn = p.src_field >= 0 ? p.jsrc[n] : T(0);
  int d, side, q, mask = 0;
  out[0] = a.eold(EX);
  out[1] = a.eold(EY);
  out[2] = a.eold(EZ);
  // Ex: i in (ib, ie), j in [jb, je), k in [kb, ke)         :43-50
  if (i > p.ib && i < p.ie && j >= p.jb && j < p.je && k >= p.kb && k < p.ke) {
    const T cb = a.cb(0);
    const T dhz = A::sub(a.h(HZ, 0, 1, 0), a.h(HZ, 0, 0, 0));
    const T hy1 = a.h(HY, 0, 0, 1), hy0 = a.h(HY, 0, 0, 0);
    const T dhy = A::sub(hy1, hy0);
    T e = A::add(out[0], A::mul(cb, A::sub(A::div(dhz, p.kd[1][j], p.rkd[1][j]),
                                            A::div(dhy, p.kd[2][k], p.rkd[2][k]))));
    if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_ex_yinc :113-123
      const long long o = psi_idx3(p, AY, i, d, k);
      T v = A::add(A::mul(p.be[q], p.psi[EX][AY][side][o]), A::div(A::mul(p.ce[q], dhz), p.dx, p.rdx));
      if (own) p.psin[EX][AY][side][o] = v;
      e = A::add(e, A::mul(cb, v));
    }
    if ((q = e_slab(k, p.kb, p.ke, P, d, side)) >= 0) {  // update_pml_ex_zinc :126-136
      T h1 = hy1, h0 = hy0;
      if (p.src_field == HY) {  // the Hy source lands between the E curl and the E-CPML
        if (in_src(p, HY, i, j, k + 1)) h1 = A::sub(h1, Jn);
        if (in_src(p, HY, i, j, k)) h0 = A::sub(h0, Jn);
      }
      const long long o = psi_idx3(p, AZ, i, j, d);
      T v = A::add(A::mul(p.be[q], p.psi[EX][AZ][side][o]), A::div(A::mul(p.ce[q], A::sub(h1, h0)), p.dx, p.rdx));
      if (own) p.psin[EX][AZ][side][o] = v;
      e = A::sub(e, A::mul(cb, v));
    }
    out[0] = e;
    mask |= 1;
  }
  // Ey: i in [ib, ie), j in (jb, je), k in [kb, ke)         :53-60
  if (i >= p.ib && i < p.ie && j > p.jb && j < p.je && k >= p.kb && k < p.ke) {
    const T cb = a.cb(1);
    const T dhx = A::sub(a.h(HX, 0, 0, 1), a.h(HX, 0, 0, 0));
    const T dhz = A::sub(a.h(HZ, 1, 0, 0), a.h(HZ, 0, 0, 0));
    T e = A::add(out[1], A::mul(cb, A::sub(A::div(dhx, p.kd[2][k], p.rkd[2][k]),
                                            A::div(dhz, p.kd[0][i], p.rkd[0][i]))));
    if (in_src(p, EY, i, j, k)) e = A::sub(e, Jn);       // update_source :104-110
    if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_ey_xinc :139-149
      const long long o = psi_idx3(p, AX, d, j, k);
      T v = A::add(A::mul(p.be[q], p.psi[EY][AX][side][o]), A::div(A::mul(p.ce[q], dhz), p.dx, p.rdx));
      if (own) p.psin[EY][AX][side][o] = v;
      e = A::sub(e, A::mul(cb, v));
    }
    if ((q = e_slab(k, p.kb, p.ke, P, d, side)) >= 0) {  // update_pml_ey_zinc :152-162
      const long long o = psi_idx3(p, AZ, i, j, d);
      T v = A::add(A::mul(p.be[q], p.psi[EY][AZ][side][o]), A::div(A::mul(p.ce[q], dhx), p.dx, p.rdx));
      if (own) p.psin[EY][AZ][side][o] = v;
      e = A::add(e, A::mul(cb, v));
    }
    out[1] = e;
    mask |= 2;
  }
  // Ez: i in [ib, ie), j in [jb, je), k in (kb, ke)         :63-70
  if (i >= p.ib && i < p.ie && j >= p.jb && j < p.je && k > p.kb && k < p.ke) {
    const T cb = a.cb(2);
    const T hy1 = a.h(HY, 1, 0, 0), hy0 = a.h(HY, 0, 0, 0);
    const T dhy = A::sub(hy1, hy0);
    const T dhx = A::sub(a.h(HX, 0, 1, 0), a.h(HX, 0, 0, 0));
    T e = A::add(out[2], A::mul(cb, A::sub(A::div(dhy, p.kd[0][i], p.rkd[0][i]),
                                            A::div(dhx, p.kd[1][j], p.rkd[1][j]))));
    if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_ez_xinc :165-175
      T h1 = hy1, h0 = hy0;
      if (p.src_field == HY) {
        if (in_src(p, HY, i + 1, j, k)) h1 = A::sub(h1, Jn);
        if (in_src(p, HY, i, j, k)) h0 = A::sub(h0, Jn);
      }
      const long long o = psi_idx3(p, AX, d, j, k);
      T v = A::add(A::mul(p.be[q], p.psi[EZ][AX][side][o]), A::div(A::mul(p.ce[q], A::sub(h1, h0)), p.dx, p.rdx));
      if (own) p.psin[EZ][AX][side][o] = v;
      e = A::add(e, A::mul(cb, v));
    }
    if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_ez_yinc :178-188
      const long long o = psi_idx3(p, AY, i, d, k);
      T v = A::add(A::mul(p.be[q], p.psi[EZ][AY][side][o]), A::div(A::mul(p.ce[q], dhx), p.dx, p.rdx));
      if (own) p.psin[EZ][AY][side][o] = v;
      e = A::sub(e, A::mul(cb, v));
    }
    out[2] = e;
    mask |= 4;
  }
  return mask;
}

// New H at cell (i, j, k) -> out[0..2] = Hx, Hy, Hz; CPML psi of H is owned by
// the cell and updated in place.
template <typename T, bool EXACT, class Acc>
__device__ __forceinline__ int y3_h_compute(const Params<T> &p, const Acc &a, int i, int j, int k, int n, T out[3]) {
  using A = Ar<T, EXACT>;
  const int P = p.P;
  const T db = p.db;
  int d, side, q, mask = 0;
  out[0] = a.hold(HX);
  out[1] = a.hold(HY);
  out[2] = a.hold(HZ);
  // Hx: i in [ib, ie), j in (jb, je), k in (kb, ke)         :73-80
  if (i >= p.ib && i < p.ie && j > p.jb && j < p.je && k > p.kb && k < p.ke) {
    const T dey = A::sub(a.e(EY, 0, 0, 0), a.e(EY, 0, 0, -1));
    const T dez = A::sub(a.e(EZ, 0, 0, 0), a.e(EZ, 0, -1, 0));
    T h = A::add(out[0], A::mul(db, A::sub(A::div(dey, p.kd[5][k], p.rkd[5][k]),
                                            A::div(dez, p.kd[4][j], p.rkd[4][j]))));
    if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_hx_yinc :191-201
      T *ps = p.psi[HX][AY][side] + psi_idx3(p, AY, i, d, k);
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dez), p.dx, p.rdx));
      *ps = v;
      h = A::sub(h, A::mul(db, v));
    }
    if ((q = h_slab(k, p.kb, p.ke, P, d, side)) >= 0) {  // update_pml_hx_zinc :204-214
      T *ps = p.psi[HX][AZ][side] + psi_idx3(p, AZ, i, j, d);
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dey), p.dx, p.rdx));
      *ps = v;
      h = A::add(h, A::mul(db, v));
    }
    out[0] = h;
    mask |= 1;
  }
  // Hy: i in (ib, ie), j in [jb, je), k in (kb, ke)         :83-90
  if (i > p.ib && i < p.ie && j >= p.jb && j < p.je && k > p.kb && k < p.ke) {
    const T dez = A::sub(a.e(EZ, 0, 0, 0), a.e(EZ, -1, 0, 0));
    const T dex = A::sub(a.e(EX, 0, 0, 0), a.e(EX, 0, 0, -1));
    T h = out[1];
    if (in_src(p, HY, i, j, k)) h = A::sub(h, p.jsrc[n]);  // source precedes update_hy
    h = A::add(h, A::mul(db, A::sub(A::div(dez, p.kd[3][i], p.rkd[3][i]),
                                     A::div(dex, p.kd[5][k], p.rkd[5][k]))));
    if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_hy_xinc :217-227
      T *ps = p.psi[HY][AX][side] + psi_idx3(p, AX, d, j, k);
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dez), p.dx, p.rdx));
      *ps = v;
      h = A::add(h, A::mul(db, v));
    }
    if ((q = h_slab(k, p.kb, p.ke, P, d, side)) >= 0) {  // update_pml_hy_zinc :230-240
      T *ps = p.psi[HY][AZ][side] + psi_idx3(p, AZ, i, j, d);
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dex), p.dx, p.rdx));
      *ps = v;
      h = A::sub(h, A::mul(db, v));
    }
    out[1] = h;
    mask |= 2;
  }
  // Hz: i in (ib, ie), j in (jb, je), k in [kb, ke)         :93-100
  if (i > p.ib && i < p.ie && j > p.jb && j < p.je && k >= p.kb && k < p.ke) {
    const T dex = A::sub(a.e(EX, 0, 0, 0), a.e(EX, 0, -1, 0));
    const T dey = A::sub(a.e(EY, 0, 0, 0), a.e(EY, -1, 0, 0));
    T h = A::add(out[2], A::mul(db, A::sub(A::div(dex, p.kd[4][j], p.rkd[4][j]),
                                            A::div(dey, p.kd[3][i], p.rkd[3][i]))));
    if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_hz_xinc :243-253
      T *ps = p.psi[HZ][AX][side] + psi_idx3(p, AX, d, j, k);
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dey), p.dx, p.rdx));
      *ps = v;
      h = A::sub(h, A::mul(db, v));
    }
    if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_hz_yinc :256-266
      T *ps = p.psi[HZ][AY][side] + psi_idx3(p, AY, i, d, k);
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dex), p.dx, p.rdx));
      *ps = v;
      h = A::add(h, A::mul(db, v));
    }
    out[2] = h;
    mask |= 4;
  }
  return mask;
}

// Port-plane capture of the raw samples the DFT fold colocates (3D slots:
// 0 Ex(kc) 1 Ey(kc) 2 Hx(kc) 3 Hx(kc+1) 4 Hy(kc) 5 Hy(kc+1)).
template <typename T>
__device__ __forceinline__ void y3_capture_e(const Params<T> &p, int s, int i, int j, int k, int mask, const T e[3]) {
  const long long pc = (long long)i * p.ny + j;
  for (int q = 0; q < 2; ++q)
    if (k == p.port_pos[q]) {
      if (mask & 1) capture(p, s, q, 0, pc, e[0]);
      if (mask & 2) capture(p, s, q, 1, pc, e[1]);
    }
}
template <typename T>
__device__ __forceinline__ void y3_capture_h(const Params<T> &p, int s, int i, int j, int k, int mask, const T h[3]) {
  const long long pc = (long long)i * p.ny + j;
  for (int q = 0; q < 2; ++q) {
    if (k == p.port_pos[q]) {
      if (mask & 1) capture(p, s, q, 2, pc, h[0]);
      if (mask & 2) capture(p, s, q, 4, pc, h[1]);
    }
    if (k == p.port_pos[q] + 1) {
      if (mask & 1) capture(p, s, q, 3, pc, h[0]);
      if (mask & 2) capture(p, s, q, 5, pc, h[1]);
    }
  }
}

// Per-cell launches (in place): E half then H half.
template <typename T, bool EXACT>
__device__ __forceinline__ void y3_e_cell(const Params<T> &p, int i, int j, int k, int n, int s) {
  const long long sy = p.nzp, sx = (long long)p.ny * p.nzp;
  const long long c = i * sx + j * sy + k;
  GlobalAcc3<T> a{p, c, sy, sx};
  T e[3];
  const int m = y3_e_compute<T, EXACT>(p, a, i, j, k, n, true, e);
  if (m & 1) p.f[EX][c] = e[0];
  if (m & 2) p.f[EY][c] = e[1];
  if (m & 4) p.f[EZ][c] = e[2];
  y3_capture_e(p, s, i, j, k, m, e);
}

template <typename T, bool EXACT, bool CG = false>
__device__ __forceinline__ void y3_h_cell(const Params<T> &p, int i, int j, int k, int n, int s) {
  const long long sy = p.nzp, sx = (long long)p.ny * p.nzp;
  const long long c = i * sx + j * sy + k;
  GlobalAcc3<T, CG> a{p, c, sy, sx};
  T h[3];
  const int m = y3_h_compute<T, EXACT>(p, a, i, j, k, n, h);
  if (m & 1) p.f[HX][c] = h[0];
  if (m & 2) p.f[HY][c] = h[1];
  if (m & 4) p.f[HZ][c] = h[2];
  y3_capture_h(p, s, i, j, k, m, h);
}

// E update of one cell (i, j, k) of a block away from the source box: the
// three curl updates, then the CPML terms -- x and y slabs uniform over a
// warp of 32 consecutive k, z slab per lane -- each component stored where its
// (i, j, k) range holds (operation order as y3_e_compute, which it equals cell
// by cell).  Nothing is updated outside [ib, ie) x [jb, je); inside, every
// neighbour read stays inside the grid arrays.  Grid arrays are addressed as
// a per-plane base plus a 32-bit offset inside the plane (plan_job rejects
// grids whose plane or slab sizes would not fit).
template <typename T, bool EXACT>
__device__ __forceinline__ void y3_e_masked(const Params<T> &p, int i, int j, int k, int s) {
  const int P = p.P;
  // nothing is updated outside [ib, ie) x [jb, je); inside, every neighbour
  // read below stays inside the grid arrays
  if (i < p.ib || i >= p.ie || j < p.jb || j >= p.je || k >= p.nz) return;
  using A = Ar<T, EXACT>;
  const int sy = p.nzp, nz = p.nz;
  const long long sx = (long long)p.ny * p.nzp, bi = i * sx;
  const int o = j * sy + k;  // offset inside the plane
  const T *const hx = p.f[HX] + bi, *const hy = p.f[HY] + bi, *const hz = p.f[HZ] + bi;
  const T hx0 = __ldg(hx + o), hy0 = __ldg(hy + o), hz0 = __ldg(hz + o);
  const T dhz_y = A::sub(__ldg(hz + (o + sy)), hz0), dhy_z = A::sub(__ldg(hy + (o + 1)), hy0);
  const T dhx_z = A::sub(__ldg(hx + (o + 1)), hx0), dhz_x = A::sub(__ldg(hz + sx + o), hz0);
  const T dhy_x = A::sub(__ldg(hy + sx + o), hy0), dhx_y = A::sub(__ldg(hx + (o + sy)), hx0);
  const T rkx = p.rkd[0][i], rky = p.rkd[1][j], rkz = p.rkd[2][k];
  const T kx = EXACT ? p.kd[0][i] : T(0), ky = EXACT ? p.kd[1][j] : T(0), kz = EXACT ? p.kd[2][k] : T(0);
  const T cb0 = __ldg(p.cb[0] + bi + o), cb1 = __ldg(p.cb[1] + bi + o), cb2 = __ldg(p.cb[2] + bi + o);
  T *const ex = p.f[EX] + bi, *const ey = p.f[EY] + bi, *const ez = p.f[EZ] + bi;
  T e[3];
  e[0] = A::add(ex[o], A::mul(cb0, A::sub(A::div(dhz_y, ky, rky), A::div(dhy_z, kz, rkz))));
  e[1] = A::add(ey[o], A::mul(cb1, A::sub(A::div(dhx_z, kz, rkz), A::div(dhz_x, kx, rkx))));
  e[2] = A::add(ez[o], A::mul(cb2, A::sub(A::div(dhy_x, kx, rkx), A::div(dhx_y, ky, rky))));
  // updated components: Ex i (ib,ie) j [jb,je) k [kb,ke); Ey i [ib,ie) j (jb,je) k [kb,ke);
  // Ez i [ib,ie) j [jb,je) k (kb,ke)
  const bool kc = k >= p.kb && k < p.ke, ko = k > p.kb && k < p.ke;
  const bool mex = i > p.ib && kc, mey = j > p.jb && kc, mez = ko;
  int d, side, q;
  if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_ey_xinc, update_pml_ez_xinc
    const int oa = (d * p.ny + j) * p.psx + k;
    if (mey) {
      T *const py = p.psi[EY][AX][side] + oa;
      const T vy = A::add(A::mul(p.be[q], *py), A::div(A::mul(p.ce[q], dhz_x), p.dx, p.rdx));
      *py = vy;
      e[1] = A::sub(e[1], A::mul(cb1, vy));
    }
    if (mez) {
      T *const pz = p.psi[EZ][AX][side] + oa;
      const T vz = A::add(A::mul(p.be[q], *pz), A::div(A::mul(p.ce[q], dhy_x), p.dx, p.rdx));
      *pz = vz;
      e[2] = A::add(e[2], A::mul(cb2, vz));
    }
  }
  if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_ex_yinc, update_pml_ez_yinc
    const int oa = (i * P + d) * p.psy + k;
    if (mex) {
      T *const px = p.psi[EX][AY][side] + oa;
      const T vx = A::add(A::mul(p.be[q], *px), A::div(A::mul(p.ce[q], dhz_y), p.dx, p.rdx));
      *px = vx;
      e[0] = A::add(e[0], A::mul(cb0, vx));
    }
    if (mez) {
      T *const pz = p.psi[EZ][AY][side] + oa;
      const T vz = A::add(A::mul(p.be[q], *pz), A::div(A::mul(p.ce[q], dhx_y), p.dx, p.rdx));
      *pz = vz;
      e[2] = A::sub(e[2], A::mul(cb2, vz));
    }
  }
  if (kc && (q = e_slab(k, p.kb, p.ke, P, d, side)) >= 0) {  // update_pml_ex_zinc, update_pml_ey_zinc
    const int oa = (i * p.ny + j) * p.psz + d;
    if (mex) {
      T *const px = p.psi[EX][AZ][side] + oa;
      const T vx = A::add(A::mul(p.be[q], *px), A::div(A::mul(p.ce[q], dhy_z), p.dx, p.rdx));
      *px = vx;
      e[0] = A::sub(e[0], A::mul(cb0, vx));
    }
    if (mey) {
      T *const py = p.psi[EY][AZ][side] + oa;
      const T vy = A::add(A::mul(p.be[q], *py), A::div(A::mul(p.ce[q], dhx_z), p.dx, p.rdx));
      *py = vy;
      e[1] = A::add(e[1], A::mul(cb1, vy));
    }
  }
  if (mex) ex[o] = e[0];
  if (mey) ey[o] = e[1];
  if (mez) ez[o] = e[2];
  if (k == p.port_pos[0] || k == p.port_pos[1])
    y3_capture_e(p, s, i, j, k, (mex ? 1 : 0) | (mey ? 2 : 0) | (mez ? 4 : 0), e);
}

// H update of one cell (i, j, k) away from the source box (as y3_h_compute;
// ib, jb >= 1, so every neighbour read stays inside the grid arrays).
template <typename T, bool EXACT, bool CG = false>
__device__ __forceinline__ void y3_h_masked(const Params<T> &p, int i, int j, int k, int s) {
  const int P = p.P;
  // nothing is updated outside [ib, ie) x [jb, je); inside, every neighbour
  // read below stays inside the grid arrays (ib, jb >= 1)
  if (i < p.ib || i >= p.ie || j < p.jb || j >= p.je || k >= p.nz) return;
  using A = Ar<T, EXACT>;
  const int sy = p.nzp, nz = p.nz;
  const long long sx = (long long)p.ny * p.nzp, bi = i * sx;
  const int o = j * sy + k;  // offset inside the plane
  const T *const ex = p.f[EX] + bi, *const ey = p.f[EY] + bi, *const ez = p.f[EZ] + bi;
  // updated components: Hx i [ib,ie) j (jb,je) k (kb,ke); Hy i (ib,ie) j [jb,je) k (kb,ke);
  // Hz i (ib,ie) j (jb,je) k [kb,ke)
  const bool ko = k > p.kb && k < p.ke, kc = k >= p.kb && k < p.ke;
  const bool mhx = j > p.jb && ko, mhy = i > p.ib && ko, mhz = i > p.ib && j > p.jb && kc;
  const T ex0 = ld_e<CG>(ex + o), ey0 = ld_e<CG>(ey + o), ez0 = ld_e<CG>(ez + o);
  // (k - 1 is read only where k > kb >= 1)
  const T dey_z = A::sub(ey0, ko ? ld_e<CG>(ey + (o - 1)) : ey0), dez_y = A::sub(ez0, ld_e<CG>(ez + (o - sy)));
  const T dez_x = A::sub(ez0, ld_e<CG>(ez - sx + o)), dex_z = A::sub(ex0, ko ? ld_e<CG>(ex + (o - 1)) : ex0);
  const T dex_y = A::sub(ex0, ld_e<CG>(ex + (o - sy))), dey_x = A::sub(ey0, ld_e<CG>(ey - sx + o));
  const T rkx = p.rkd[3][i], rky = p.rkd[4][j], rkz = p.rkd[5][k];
  const T kx = EXACT ? p.kd[3][i] : T(0), ky = EXACT ? p.kd[4][j] : T(0), kz = EXACT ? p.kd[5][k] : T(0);
  const T db = p.db;
  T *const hx = p.f[HX] + bi, *const hy = p.f[HY] + bi, *const hz = p.f[HZ] + bi;
  T h[3];
  h[0] = A::add(hx[o], A::mul(db, A::sub(A::div(dey_z, kz, rkz), A::div(dez_y, ky, rky))));
  h[1] = A::add(hy[o], A::mul(db, A::sub(A::div(dez_x, kx, rkx), A::div(dex_z, kz, rkz))));
  h[2] = A::add(hz[o], A::mul(db, A::sub(A::div(dex_y, ky, rky), A::div(dey_x, kx, rkx))));
  int d, side, q;
  if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {  // update_pml_hy_xinc, update_pml_hz_xinc
    const int oa = (d * p.ny + j) * p.psx + k;
    if (mhy) {
      T *const py = p.psi[HY][AX][side] + oa;
      const T vy = A::add(A::mul(p.bh[q], *py), A::div(A::mul(p.ch[q], dez_x), p.dx, p.rdx));
      *py = vy;
      h[1] = A::add(h[1], A::mul(db, vy));
    }
    if (mhz) {
      T *const pz = p.psi[HZ][AX][side] + oa;
      const T vz = A::add(A::mul(p.bh[q], *pz), A::div(A::mul(p.ch[q], dey_x), p.dx, p.rdx));
      *pz = vz;
      h[2] = A::sub(h[2], A::mul(db, vz));
    }
  }
  if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {  // update_pml_hx_yinc, update_pml_hz_yinc
    const int oa = (i * P + d) * p.psy + k;
    if (mhx) {
      T *const px = p.psi[HX][AY][side] + oa;
      const T vx = A::add(A::mul(p.bh[q], *px), A::div(A::mul(p.ch[q], dez_y), p.dx, p.rdx));
      *px = vx;
      h[0] = A::sub(h[0], A::mul(db, vx));
    }
    if (mhz) {
      T *const pz = p.psi[HZ][AY][side] + oa;
      const T vz = A::add(A::mul(p.bh[q], *pz), A::div(A::mul(p.ch[q], dex_y), p.dx, p.rdx));
      *pz = vz;
      h[2] = A::add(h[2], A::mul(db, vz));
    }
  }
  if (ko && (q = h_slab(k, p.kb, p.ke, P, d, side)) >= 0) {  // update_pml_hx_zinc, update_pml_hy_zinc
    const int oa = (i * p.ny + j) * p.psz + d;
    if (mhx) {
      T *const px = p.psi[HX][AZ][side] + oa;
      const T vx = A::add(A::mul(p.bh[q], *px), A::div(A::mul(p.ch[q], dey_z), p.dx, p.rdx));
      *px = vx;
      h[0] = A::add(h[0], A::mul(db, vx));
    }
    if (mhy) {
      T *const py = p.psi[HY][AZ][side] + oa;
      const T vy = A::add(A::mul(p.bh[q], *py), A::div(A::mul(p.ch[q], dex_z), p.dx, p.rdx));
      *py = vy;
      h[1] = A::sub(h[1], A::mul(db, vy));
    }
  }
  if (mhx) hx[o] = h[0];
  if (mhy) hy[o] = h[1];
  if (mhz) hz[o] = h[2];
  if (k == p.port_pos[0] || k == p.port_pos[1] || k == p.port_pos[0] + 1 || k == p.port_pos[1] + 1)
    y3_capture_h(p, s, i, j, k, (mhx ? 1 : 0) | (mhy ? 2 : 0) | (mhz ? 4 : 0), h);
}

// ---------------------------------------------------------------------------
// 2D TM (FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_funcs.py)
// psi arrays: x-slab [P][ny], y-slab [nx][P].
// ---------------------------------------------------------------------------
template <typename T, bool EXACT>
__device__ __forceinline__ void tm2_e_cell(const Params<T> &p, int i, int j, int n, int s) {
  using A = Ar<T, EXACT>;
  const int ny = p.ny, P = p.P;
  const long long c = (long long)i * ny + j;
  const T *Hx = p.f[HX], *Hy = p.f[HY];
  int d, side, q;
  if (i >= p.ib && i < p.ie && j >= p.jb && j < p.je) {  // update_ez :44-49
    const T cb = p.cb[2][c];
    const T dhy = A::sub(Hy[c + ny], Hy[c]);
    const T dhx = A::sub(Hx[c + 1], Hx[c]);
    T e = A::add(p.f[EZ][c], A::mul(cb, A::sub(A::div(dhy, p.kd[0][i], p.rkd[0][i]),
                                                A::div(dhx, p.kd[1][j], p.rkd[1][j]))));
    if (in_src(p, EZ, i, j, 0)) e = A::sub(e, p.jsrc[n]);  // update_source :71-76
    if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {    // update_pml_ez_xinc :80-88
      T *ps = p.psi[EZ][AX][side] + (long long)d * ny + j;
      T v = A::add(A::mul(p.be[q], *ps), A::div(A::mul(p.ce[q], dhy), p.dx, p.rdx));
      *ps = v;
      e = A::add(e, A::mul(cb, v));
    }
    if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {    // update_pml_ez_yinc :92-100
      T *ps = p.psi[EZ][AY][side] + (long long)i * P + d;
      T v = A::add(A::mul(p.be[q], *ps), A::div(A::mul(p.ce[q], dhx), p.dx, p.rdx));
      *ps = v;
      e = A::sub(e, A::mul(cb, v));
    }
    p.f[EZ][c] = e;
    if (i == p.port_pos[0]) capture(p, s, 0, 0, j, e);
    if (i == p.port_pos[1]) capture(p, s, 1, 0, j, e);
  }
}

template <typename T, bool EXACT>
__device__ __forceinline__ void tm2_h_cell(const Params<T> &p, int i, int j, int n, int s) {
  using A = Ar<T, EXACT>;
  const int ny = p.ny, P = p.P;
  const long long c = (long long)i * ny + j;
  const T *Ez = p.f[EZ];
  const T db = p.db;
  int d, side, q;
  if (i >= p.ib && i < p.ie && j > p.jb && j < p.je) {  // update_hx :53-58
    const T dez = A::sub(Ez[c - 1], Ez[c]);
    T h = A::add(p.f[HX][c], A::div(A::mul(db, dez), p.kd[4][j], p.rkd[4][j]));
    if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {   // update_pml_hx_yinc :104-112
      T *ps = p.psi[HX][AY][side] + (long long)i * P + d;
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], A::sub(Ez[c], Ez[c - 1])), p.dx, p.rdx));
      *ps = v;
      h = A::sub(h, A::mul(db, v));
    }
    p.f[HX][c] = h;
  }
  if (i > p.ib && i < p.ie && j >= p.jb && j < p.je) {  // update_hy :62-67
    const T dez = A::sub(Ez[c], Ez[c - ny]);
    T h = A::add(p.f[HY][c], A::div(A::mul(db, dez), p.kd[3][i], p.rkd[3][i]));
    if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {   // update_pml_hy_xinc :116-124
      T *ps = p.psi[HY][AX][side] + (long long)d * ny + j;
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dez), p.dx, p.rdx));
      *ps = v;
      h = A::add(h, A::mul(db, v));
    }
    p.f[HY][c] = h;
    if (i == p.port_pos[0]) capture(p, s, 0, 1, j, h);
    if (i == p.port_pos[1]) capture(p, s, 1, 1, j, h);
    if (i == p.port_pos[0] + 1) capture(p, s, 0, 2, j, h);
    if (i == p.port_pos[1] + 1) capture(p, s, 1, 2, j, h);
  }
}

// ---------------------------------------------------------------------------
// 2D TE (FDTD/GPU/FDTD_2D_TE/s-parameter_extraction/fdtd_funcs.py)
// ---------------------------------------------------------------------------
template <typename T, bool EXACT>
__device__ __forceinline__ void te2_e_cell(const Params<T> &p, int i, int j, int n, int s) {
  using A = Ar<T, EXACT>;
  const int ny = p.ny, P = p.P;
  const long long c = (long long)i * ny + j;
  const T *Hz = p.f[HZ];
  int d, side, q;
  if (i > p.ib && i < p.ie && j >= p.jb && j < p.je) {  // update_ex :43-49
    const T cb = p.cb[0][c];
    const T dhz = A::sub(Hz[c + 1], Hz[c]);
    T e = A::add(p.f[EX][c], A::div(A::mul(cb, dhz), p.kd[1][j], p.rkd[1][j]));
    if ((q = e_slab(j, p.jb, p.je, P, d, side)) >= 0) {   // update_pml_ex_yinc :79-87
      T *ps = p.psi[EX][AY][side] + (long long)i * P + d;
      T v = A::add(A::mul(p.be[q], *ps), A::div(A::mul(p.ce[q], dhz), p.dx, p.rdx));
      *ps = v;
      e = A::add(e, A::mul(cb, v));
    }
    p.f[EX][c] = e;
  }
  if (i >= p.ib && i < p.ie && j > p.jb && j < p.je) {  // update_ey :52-58
    const T cb = p.cb[1][c];
    T e = A::add(p.f[EY][c], A::div(A::mul(cb, A::sub(Hz[c], Hz[c + ny])), p.kd[0][i], p.rkd[0][i]));
    if ((q = e_slab(i, p.ib, p.ie, P, d, side)) >= 0) {   // update_pml_ey_xinc :91-99
      T *ps = p.psi[EY][AX][side] + (long long)d * ny + j;
      T v = A::add(A::mul(p.be[q], *ps), A::div(A::mul(p.ce[q], A::sub(Hz[c + ny], Hz[c])), p.dx, p.rdx));
      *ps = v;
      e = A::sub(e, A::mul(cb, v));
    }
    p.f[EY][c] = e;
    if (i == p.port_pos[0]) capture(p, s, 0, 0, j, e);
    if (i == p.port_pos[1]) capture(p, s, 1, 0, j, e);
  }
}

template <typename T, bool EXACT>
__device__ __forceinline__ void te2_h_cell(const Params<T> &p, int i, int j, int n, int s) {
  using A = Ar<T, EXACT>;
  const int ny = p.ny, P = p.P;
  const long long c = (long long)i * ny + j;
  const T *Ex = p.f[EX], *Ey = p.f[EY];
  const T db = p.db;
  int d, side, q;
  if (i > p.ib && i < p.ie && j > p.jb && j < p.je) {  // update_hz :61-67
    const T dex = A::sub(Ex[c], Ex[c - 1]);
    const T dey = A::sub(Ey[c], Ey[c - ny]);
    T h = A::add(p.f[HZ][c], A::mul(db, A::sub(A::div(dex, p.kd[4][j], p.rkd[4][j]),
                                                A::div(dey, p.kd[3][i], p.rkd[3][i]))));
    if (in_src(p, HZ, i, j, 0)) h = A::sub(h, p.jsrc[n]);  // source after update_hz
    if ((q = h_slab(i, p.ib, p.ie, P, d, side)) >= 0) {     // update_pml_hz_xinc :103-111
      T *ps = p.psi[HZ][AX][side] + (long long)d * ny + j;
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dey), p.dx, p.rdx));
      *ps = v;
      h = A::sub(h, A::mul(db, v));
    }
    if ((q = h_slab(j, p.jb, p.je, P, d, side)) >= 0) {     // update_pml_hz_yinc :115-123
      T *ps = p.psi[HZ][AY][side] + (long long)i * P + d;
      T v = A::add(A::mul(p.bh[q], *ps), A::div(A::mul(p.ch[q], dex), p.dx, p.rdx));
      *ps = v;
      h = A::add(h, A::mul(db, v));
    }
    p.f[HZ][c] = h;
    if (i == p.port_pos[0]) capture(p, s, 0, 1, j, h);
    if (i == p.port_pos[1]) capture(p, s, 1, 1, j, h);
    if (i == p.port_pos[0] + 1) capture(p, s, 0, 2, j, h);
    if (i == p.port_pos[1] + 1) capture(p, s, 1, 2, j, h);
  }
}

}  // namespace oidt
