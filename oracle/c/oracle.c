/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C, float64 (or float32), OpenMP
 * restatement of the reference's S-parameter time loop, used as the timed CPU
 * baseline and cross-checked bit for bit against the NumPy oracle
 * (oracle/fdtd_ref.py).  Never linked into the product.
 *
 * Per time step, in the reference's launch order:
 *   2D TM  FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_main.py:275-304
 *          (kernels fdtd_funcs.py:43-144)
 *   3D     FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_main.py:357-406
 *          (kernels fdtd_funcs.py:43-292)
 * Build with -ffp-contract=off so no multiply-add is fused: every operation
 * rounds exactly as the reference's float64 run does.
 */
#include <stddef.h>
#include <stdint.h>

/* Field, coefficient and psi type: double (the parity oracle) or, built with
 * -DORACLE_REAL=float, float (the CPU timing at the reference's default
 * float32 precision).  DFT accumulators and twiddles are double in both. */
#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
typedef ORACLE_REAL real;

typedef struct {
  int nx, ny, nz, P, ib, jb, kb, ie, je, ke;
  real *f[6];            /* EX EY EZ HX HY HZ (reference layout) */
  const real *cb[3];     /* CBX CBY CBZ */
  const real *kd[6];     /* kxe kye kze kxh kyh kzh */
  const real *be, *ce, *bh, *ch;
  real db, dx;
  real *psi[6][3][2];    /* [field][axis][lo/hi] */
  int src_field, slo[3], shi[3];
  const real *jsrc;
  int port[2];
  int nf, nt;
  const double *tw[4];   /* cosE sinE cosH sinH [nf][nt] */
  double *dft[2][4][2];  /* [port][comp][re/im]: 3D [nf][nx][ny], 2D [nf][ny] */
} OracleState;

#define IDX3(i, j, k) (((long long)(i) * ny + (j)) * nz + (k))
enum { EX, EY, EZ, HX, HY, HZ };

static void src3(OracleState *s, int n) {
  if (s->src_field < 0) return;
  const int ny = s->ny, nz = s->nz;
  real *F = s->f[s->src_field];
  const real J = s->jsrc[n];
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = s->slo[0]; i < s->shi[0]; ++i)
    for (int j = s->slo[1]; j < s->shi[1]; ++j)
      for (int k = s->slo[2]; k < s->shi[2]; ++k) F[IDX3(i, j, k)] = F[IDX3(i, j, k)] - J;
}

/* E-field CPML along `axis` for field E using the H difference along that
 * axis; t0/t1 give the transverse ranges (as [lo, hi) per axis, the slab axis
 * entry ignored).  sign +1: E + cb psi, -1: E - cb psi. */
static void pml_e3(OracleState *s, int fe, int fh, int axis, int sign, const real *cb, const int lo[3],
                   const int hi[3]) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, P = s->P;
  const int b = axis == 0 ? s->ib : axis == 1 ? s->jb : s->kb;
  const int e = axis == 0 ? s->ie : axis == 1 ? s->je : s->ke;
  real *E = s->f[fe];
  const real *H = s->f[fh];
  int r0[3] = {lo[0], lo[1], lo[2]}, r1[3] = {hi[0], hi[1], hi[2]};
  r0[axis] = 0;
  r1[axis] = P;
  const long long st = axis == 0 ? (long long)ny * nz : axis == 1 ? nz : 1;
  const int pd[3] = {axis == 0 ? P : nx, axis == 1 ? P : ny, axis == 2 ? P : nz};
  for (int side = 0; side < 2; ++side) {
    real *ps = s->psi[fe][axis][side];
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = r0[0]; i < r1[0]; ++i)
      for (int j = r0[1]; j < r1[1]; ++j)
        for (int k = r0[2]; k < r1[2]; ++k) {
          const int d = axis == 0 ? i : axis == 1 ? j : k;
          int c[3] = {i, j, k};
          c[axis] = side == 0 ? b + d : e - P + d;
          const int q = side == 0 ? P - 1 - d : d;
          const long long cc = IDX3(c[0], c[1], c[2]);
          const long long pi = ((long long)i * pd[1] + j) * pd[2] + k;
          ps[pi] = s->be[q] * ps[pi] + s->ce[q] * (H[cc + st] - H[cc]) / s->dx;
          if (sign > 0)
            E[cc] = E[cc] + cb[cc] * ps[pi];
          else
            E[cc] = E[cc] - cb[cc] * ps[pi];
        }
  }
}

/* H-field CPML: slab index d in 1..P-1; low coefficient P-d, high d. */
static void pml_h3(OracleState *s, int fh, int fe, int axis, int sign, const int lo[3], const int hi[3]) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, P = s->P;
  const int b = axis == 0 ? s->ib : axis == 1 ? s->jb : s->kb;
  const int e = axis == 0 ? s->ie : axis == 1 ? s->je : s->ke;
  real *H = s->f[fh];
  const real *E = s->f[fe];
  int r0[3] = {lo[0], lo[1], lo[2]}, r1[3] = {hi[0], hi[1], hi[2]};
  r0[axis] = 1;
  r1[axis] = P;
  const long long st = axis == 0 ? (long long)ny * nz : axis == 1 ? nz : 1;
  const int pd[3] = {axis == 0 ? P : nx, axis == 1 ? P : ny, axis == 2 ? P : nz};
  for (int side = 0; side < 2; ++side) {
    real *ps = s->psi[fh][axis][side];
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = r0[0]; i < r1[0]; ++i)
      for (int j = r0[1]; j < r1[1]; ++j)
        for (int k = r0[2]; k < r1[2]; ++k) {
          const int d = axis == 0 ? i : axis == 1 ? j : k;
          int c[3] = {i, j, k};
          c[axis] = side == 0 ? b + d : e - P + d;
          const int q = side == 0 ? P - d : d;
          const long long cc = IDX3(c[0], c[1], c[2]);
          const long long pi = ((long long)i * pd[1] + j) * pd[2] + k;
          ps[pi] = s->bh[q] * ps[pi] + s->ch[q] * (E[cc] - E[cc - st]) / s->dx;
          if (sign > 0)
            H[cc] = H[cc] + s->db * ps[pi];
          else
            H[cc] = H[cc] - s->db * ps[pi];
        }
  }
}

static void step3(OracleState *s, int n) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int ib = s->ib, jb = s->jb, kb = s->kb, ie = s->ie, je = s->je, ke = s->ke;
  real *Ex = s->f[EX], *Ey = s->f[EY], *Ez = s->f[EZ], *Hx = s->f[HX], *Hy = s->f[HY], *Hz = s->f[HZ];
  const real *kxe = s->kd[0], *kye = s->kd[1], *kze = s->kd[2], *kxh = s->kd[3], *kyh = s->kd[4], *kzh = s->kd[5];
  const long long SX = (long long)ny * nz, SY = nz;
  /* update_ex / update_ey / update_ez  (fdtd_funcs.py:43-70) */
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ib + 1; i < ie; ++i)
    for (int j = jb; j < je; ++j)
      for (int k = kb; k < ke; ++k) {
        const long long c = IDX3(i, j, k);
        Ex[c] = Ex[c] + s->cb[0][c] * ((Hz[c + SY] - Hz[c]) / kye[j] - (Hy[c + 1] - Hy[c]) / kze[k]);
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ib; i < ie; ++i)
    for (int j = jb + 1; j < je; ++j)
      for (int k = kb; k < ke; ++k) {
        const long long c = IDX3(i, j, k);
        Ey[c] = Ey[c] + s->cb[1][c] * ((Hx[c + 1] - Hx[c]) / kze[k] - (Hz[c + SX] - Hz[c]) / kxe[i]);
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ib; i < ie; ++i)
    for (int j = jb; j < je; ++j)
      for (int k = kb + 1; k < ke; ++k) {
        const long long c = IDX3(i, j, k);
        Ez[c] = Ez[c] + s->cb[2][c] * ((Hy[c + SX] - Hy[c]) / kxe[i] - (Hx[c + SY] - Hx[c]) / kye[j]);
      }
  src3(s, n);
  {
    int lo[3], hi[3];
    /* E-CPML, launch order fdtd_main.py:382-387 */
    lo[0] = ib + 1; hi[0] = ie; lo[1] = 0; hi[1] = 0; lo[2] = kb; hi[2] = ke;
    pml_e3(s, EX, HZ, 1, +1, s->cb[0], lo, hi);
    lo[0] = ib + 1; hi[0] = ie; lo[1] = jb; hi[1] = je;
    pml_e3(s, EX, HY, 2, -1, s->cb[0], lo, hi);
    lo[1] = jb + 1; hi[1] = je; lo[2] = kb; hi[2] = ke;
    pml_e3(s, EY, HZ, 0, -1, s->cb[1], lo, hi);
    lo[0] = ib; hi[0] = ie; lo[1] = jb + 1; hi[1] = je;
    pml_e3(s, EY, HX, 2, +1, s->cb[1], lo, hi);
    lo[1] = jb; hi[1] = je; lo[2] = kb + 1; hi[2] = ke;
    pml_e3(s, EZ, HY, 0, +1, s->cb[2], lo, hi);
    lo[0] = ib; hi[0] = ie; lo[2] = kb + 1; hi[2] = ke;
    pml_e3(s, EZ, HX, 1, -1, s->cb[2], lo, hi);
  }
  /* update_hx / update_hy / update_hz  (fdtd_funcs.py:73-100) */
  const real db = s->db;
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ib; i < ie; ++i)
    for (int j = jb + 1; j < je; ++j)
      for (int k = kb + 1; k < ke; ++k) {
        const long long c = IDX3(i, j, k);
        Hx[c] = Hx[c] + db * ((Ey[c] - Ey[c - 1]) / kzh[k] - (Ez[c] - Ez[c - SY]) / kyh[j]);
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ib + 1; i < ie; ++i)
    for (int j = jb; j < je; ++j)
      for (int k = kb + 1; k < ke; ++k) {
        const long long c = IDX3(i, j, k);
        Hy[c] = Hy[c] + db * ((Ez[c] - Ez[c - SX]) / kxh[i] - (Ex[c] - Ex[c - 1]) / kzh[k]);
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ib + 1; i < ie; ++i)
    for (int j = jb + 1; j < je; ++j)
      for (int k = kb; k < ke; ++k) {
        const long long c = IDX3(i, j, k);
        Hz[c] = Hz[c] + db * ((Ex[c] - Ex[c - SY]) / kyh[j] - (Ey[c] - Ey[c - SX]) / kxh[i]);
      }
  {
    int lo[3], hi[3];
    /* H-CPML, launch order fdtd_main.py:395-400 */
    lo[0] = ib; hi[0] = ie; lo[2] = kb + 1; hi[2] = ke; lo[1] = 0; hi[1] = 0;
    pml_h3(s, HX, EZ, 1, -1, lo, hi);
    lo[1] = jb + 1; hi[1] = je;
    pml_h3(s, HX, EY, 2, +1, lo, hi);
    lo[1] = jb; hi[1] = je; lo[2] = kb + 1; hi[2] = ke;
    pml_h3(s, HY, EZ, 0, +1, lo, hi);
    lo[0] = ib + 1; hi[0] = ie;
    pml_h3(s, HY, EX, 2, -1, lo, hi);
    lo[1] = jb + 1; hi[1] = je; lo[2] = kb; hi[2] = ke;
    pml_h3(s, HZ, EY, 0, -1, lo, hi);
    lo[0] = ib + 1; hi[0] = ie;
    pml_h3(s, HZ, EX, 1, +1, lo, hi);
  }
  /* simul_fft_efield / simul_fft_hfield at both ports (fdtd_funcs.py:269-292) */
  const int P = s->P, nf = s->nf, nt = s->nt;
  for (int q = 0; q < 2; ++q) {
    const int kc = s->port[q];
#pragma omp parallel for schedule(static)
    for (int f = 0; f < nf; ++f) {
      const double cE = s->tw[0][(long long)f * nt + n], sE = s->tw[1][(long long)f * nt + n];
      const double cH = s->tw[2][(long long)f * nt + n], sH = s->tw[3][(long long)f * nt + n];
      for (int i = P; i < nx - P; ++i)
        for (int j = P; j < ny - P; ++j) {
          const long long o = ((long long)f * nx + i) * ny + j;
          const double x = 0.5 * (Ex[IDX3(i, j, kc)] + Ex[IDX3(i + 1, j, kc)]);
          const double y = 0.5 * (Ey[IDX3(i, j, kc)] + Ey[IDX3(i, j + 1, kc)]);
          s->dft[q][0][0][o] = s->dft[q][0][0][o] + x * cE;
          s->dft[q][0][1][o] = s->dft[q][0][1][o] - x * sE;
          s->dft[q][1][0][o] = s->dft[q][1][0][o] + y * cE;
          s->dft[q][1][1][o] = s->dft[q][1][1][o] - y * sE;
        }
      for (int i = P; i < nx - P; ++i)
        for (int j = P; j < ny - P; ++j) {
          const long long o = ((long long)f * nx + i) * ny + j;
          const double x = 0.25 * (Hx[IDX3(i, j, kc)] + Hx[IDX3(i, j + 1, kc)] + Hx[IDX3(i, j, kc + 1)] +
                                   Hx[IDX3(i, j + 1, kc + 1)]);
          const double y = 0.25 * (Hy[IDX3(i, j, kc)] + Hy[IDX3(i + 1, j, kc)] + Hy[IDX3(i, j, kc + 1)] +
                                   Hy[IDX3(i + 1, j, kc + 1)]);
          s->dft[q][2][0][o] = s->dft[q][2][0][o] + x * cH;
          s->dft[q][2][1][o] = s->dft[q][2][1][o] - x * sH;
          s->dft[q][3][0][o] = s->dft[q][3][0][o] + y * cH;
          s->dft[q][3][1][o] = s->dft[q][3][1][o] - y * sH;
        }
    }
  }
}

/* 2D TM (Ez, Hx, Hy) -- FDTD_2D_TM/.../fdtd_funcs.py:43-144 */
static void step_tm2(OracleState *s, int n) {
  const int nx = s->nx, ny = s->ny, P = s->P, ib = s->ib, jb = s->jb, ie = s->ie, je = s->je;
  real *Ez = s->f[EZ], *Hx = s->f[HX], *Hy = s->f[HY];
  const real *cb = s->cb[2], *kxe = s->kd[0], *kye = s->kd[1], *kxh = s->kd[3], *kyh = s->kd[4];
  const real db = s->db, dx = s->dx;
#define I2(i, j) ((long long)(i) * ny + (j))
#pragma omp parallel for schedule(static)
  for (int i = ib; i < ie; ++i)
    for (int j = jb; j < je; ++j) {
      const long long c = I2(i, j);
      Ez[c] = Ez[c] + cb[c] * ((Hy[c + ny] - Hy[c]) / kxe[i] - (Hx[c + 1] - Hx[c]) / kye[j]);
    }
  if (s->src_field == EZ)
    for (int i = s->slo[0]; i < s->shi[0]; ++i)
      for (int j = s->slo[1]; j < s->shi[1]; ++j) Ez[I2(i, j)] = Ez[I2(i, j)] - s->jsrc[n];
  {
    real *lo = s->psi[EZ][0][0], *hi = s->psi[EZ][0][1];
    for (int i = 0; i < P; ++i)
      for (int j = jb; j < je; ++j) {
        long long c = I2(ib + i, j), p = (long long)i * ny + j;
        lo[p] = s->be[P - 1 - i] * lo[p] + s->ce[P - 1 - i] * (Hy[c + ny] - Hy[c]) / dx;
        Ez[c] = Ez[c] + cb[c] * lo[p];
        c = I2(ie - P + i, j);
        hi[p] = s->be[i] * hi[p] + s->ce[i] * (Hy[c + ny] - Hy[c]) / dx;
        Ez[c] = Ez[c] + cb[c] * hi[p];
      }
    lo = s->psi[EZ][1][0];
    hi = s->psi[EZ][1][1];
    for (int i = ib; i < ie; ++i)
      for (int j = 0; j < P; ++j) {
        long long c = I2(i, jb + j), p = (long long)i * P + j;
        lo[p] = s->be[P - 1 - j] * lo[p] + s->ce[P - 1 - j] * (Hx[c + 1] - Hx[c]) / dx;
        Ez[c] = Ez[c] - cb[c] * lo[p];
        c = I2(i, je - P + j);
        hi[p] = s->be[j] * hi[p] + s->ce[j] * (Hx[c + 1] - Hx[c]) / dx;
        Ez[c] = Ez[c] - cb[c] * hi[p];
      }
  }
#pragma omp parallel for schedule(static)
  for (int i = ib; i < ie; ++i)
    for (int j = jb + 1; j < je; ++j) {
      const long long c = I2(i, j);
      Hx[c] = Hx[c] + db * (Ez[c - 1] - Ez[c]) / kyh[j];
    }
#pragma omp parallel for schedule(static)
  for (int i = ib + 1; i < ie; ++i)
    for (int j = jb; j < je; ++j) {
      const long long c = I2(i, j);
      Hy[c] = Hy[c] + db * (Ez[c] - Ez[c - ny]) / kxh[i];
    }
  {
    real *lo = s->psi[HX][1][0], *hi = s->psi[HX][1][1];
    for (int i = ib; i < ie; ++i)
      for (int j = 1; j < P; ++j) {
        long long c = I2(i, jb + j), p = (long long)i * P + j;
        lo[p] = s->bh[P - j] * lo[p] + s->ch[P - j] * (Ez[c] - Ez[c - 1]) / dx;
        Hx[c] = Hx[c] - db * lo[p];
        c = I2(i, je - P + j);
        hi[p] = s->bh[j] * hi[p] + s->ch[j] * (Ez[c] - Ez[c - 1]) / dx;
        Hx[c] = Hx[c] - db * hi[p];
      }
    lo = s->psi[HY][0][0];
    hi = s->psi[HY][0][1];
    for (int i = 1; i < P; ++i)
      for (int j = jb; j < je; ++j) {
        long long c = I2(ib + i, j), p = (long long)i * ny + j;
        lo[p] = s->bh[P - i] * lo[p] + s->ch[P - i] * (Ez[c] - Ez[c - ny]) / dx;
        Hy[c] = Hy[c] + db * lo[p];
        c = I2(ie - P + i, j);
        hi[p] = s->bh[i] * hi[p] + s->ch[i] * (Ez[c] - Ez[c - ny]) / dx;
        Hy[c] = Hy[c] + db * hi[p];
      }
  }
  const int nf = s->nf, nt = s->nt;
  for (int q = 0; q < 2; ++q) {
    const int ic = s->port[q];
    for (int f = 0; f < nf; ++f) {
      const double cE = s->tw[0][(long long)f * nt + n], sE = s->tw[1][(long long)f * nt + n];
      const double cH = s->tw[2][(long long)f * nt + n], sH = s->tw[3][(long long)f * nt + n];
      for (int j = P; j < ny - P; ++j) {
        const long long o = (long long)f * ny + j;
        const double x = Ez[I2(ic, j)];
        s->dft[q][0][0][o] = s->dft[q][0][0][o] + x * cE;
        s->dft[q][0][1][o] = s->dft[q][0][1][o] - x * sE;
        const double y = 0.5 * (Hy[I2(ic, j)] + Hy[I2(ic + 1, j)]);
        s->dft[q][1][0][o] = s->dft[q][1][0][o] + y * cH;
        s->dft[q][1][1][o] = s->dft[q][1][1][o] - y * sH;
      }
    }
  }
#undef I2
  (void)nx;
}

/* Advance steps n0 .. n0 + count - 1.  mode: 0 = 2D TM, 2 = 3D. */
int oracle_run(OracleState *s, int mode, int n0, int count) {
  if (mode != 0 && mode != 2) return -1;
  for (int n = n0; n < n0 + count; ++n) {
    if (mode == 2)
      step3(s, n);
    else
      step_tm2(s, n);
  }
  return 0;
}

int oracle_state_size(void) { return (int)sizeof(OracleState); }
int oracle_real_size(void) { return (int)sizeof(real); }
