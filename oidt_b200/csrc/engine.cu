// engine.cu -- liboidt.so: job management, launches and the C ABI (include/oidt.h).
//
// Device layout of one job (one cudaMallocAsync block, 256-byte aligned
// sub-buffers): fields and coefficient grids in the reference layout
// ([nx][ny] or [nx][ny][nz], C order), 1-D kappa*dx arrays and their
// reciprocals, CPML psi slabs in the reference's PSI_<F>_<A><LO|HI> shapes,
// the source waveform, float64 twiddle tables [nf][nt], the capture ring
// [K][port][slot][plane] and the float64 complex DFT accumulators
// [port][comp][nf][plane].
//
// A time step is two launches (E half, H half; kernels.cuh).  Every K steps a
// fold kernel turns the K captured port planes into float64 DFT updates and a
// one-thread kernel advances the job's step counter, so a K-step block is a
// fixed launch sequence that is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/oidt.h"
#include "kernels.cuh"

using namespace oidt;

namespace {

constexpr int kDefaultRing = 32;
constexpr int kFoldF = 8;        // frequencies per fold thread
constexpr int kBlock3Z = 32, kBlock3Y = 4;
constexpr int kBlock2 = 128;

// ---------------------------------------------------------------------------
// Kernels: single-job and multi-job launches of the per-cell updates.
// ---------------------------------------------------------------------------
template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_y3_e(Params<T> p, int s) {
  const int k = blockIdx.x * kBlock3Z + threadIdx.x, j = blockIdx.y * kBlock3Y + threadIdx.y, i = blockIdx.z;
  if (k >= p.nz || j >= p.ny) return;
  y3_e_cell<T, EXACT>(p, i, j, k, p.state[0] + s, s);
}
template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_y3_h(Params<T> p, int s) {
  const int k = blockIdx.x * kBlock3Z + threadIdx.x, j = blockIdx.y * kBlock3Y + threadIdx.y, i = blockIdx.z;
  if (k >= p.nz || j >= p.ny) return;
  y3_h_cell<T, EXACT>(p, i, j, k, p.state[0] + s, s);
}
template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_2d_e(Params<T> p, int s) {
  const int j = blockIdx.x * kBlock2 + threadIdx.x, i = blockIdx.y;
  if (j >= p.ny) return;
  if (p.mode == OIDT_MODE_TM2)
    tm2_e_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
  else
    te2_e_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
}
template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_2d_h(Params<T> p, int s) {
  const int j = blockIdx.x * kBlock2 + threadIdx.x, i = blockIdx.y;
  if (j >= p.ny) return;
  if (p.mode == OIDT_MODE_TM2)
    tm2_h_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
  else
    te2_h_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
}

// Multi-job launch: block b works on tile tiles[b] = {job, i, j0, k0} of the
// job whose parameters live at params[job] (device memory).  3D tiles are
// 32 (k) x 4 (j) cells of one x-plane, 2D tiles 128 (j) cells of one x-line.
struct Tile {
  int job, i, j0, k0;
};
template <typename T, bool EXACT, bool E_HALF>
__global__ void __launch_bounds__(128) k_batch(const Params<T> *__restrict__ params,
                                               const Tile *__restrict__ tiles, int s) {
  static_assert(sizeof(Params<T>) % 8 == 0, "Params must be a whole number of 8-byte words");
  __shared__ __align__(16) unsigned long long sp[sizeof(Params<T>) / 8];
  const Tile t = tiles[blockIdx.x];
  {
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(params + t.job);
    for (int w = threadIdx.x; w < (int)(sizeof(Params<T>) / 8); w += blockDim.x) sp[w] = src[w];
  }
  __syncthreads();
  const Params<T> &p = *reinterpret_cast<const Params<T> *>(sp);
  const int n = p.state[0] + s;
  if (p.mode == OIDT_MODE_YEE3D) {
    const int k = t.k0 + (threadIdx.x & 31), j = t.j0 + (threadIdx.x >> 5);
    if (k >= p.nz || j >= p.ny) return;
    if (E_HALF)
      y3_e_cell<T, EXACT>(p, t.i, j, k, n, s);
    else
      y3_h_cell<T, EXACT>(p, t.i, j, k, n, s);
  } else {
    const int j = t.j0 + threadIdx.x;
    if (j >= p.ny) return;
    if (p.mode == OIDT_MODE_TM2) {
      if (E_HALF) tm2_e_cell<T, EXACT>(p, t.i, j, n, s); else tm2_h_cell<T, EXACT>(p, t.i, j, n, s);
    } else {
      if (E_HALF) te2_e_cell<T, EXACT>(p, t.i, j, n, s); else te2_h_cell<T, EXACT>(p, t.i, j, n, s);
    }
  }
}

// ---------------------------------------------------------------------------
// DFT fold: acc[port][comp][f][cell] += sum_s x_s(cell) * (cos, -sin)[f][n0+s]
// in float64, s = 0..count-1 in order (the reference's running sum, one step
// at a time: fdtd_funcs.py simul_fft_efield/hfield).  x_s is the colocated
// port-plane sample computed from the captured raw planes:
//   TM2 E: Ez[ic,j]                 H: (Hy[ic,j] + Hy[ic+1,j]) / 2
//   TE2 E: (Ey[ic,j] + Ey[ic,j+1])/2  H: 4-point Hz average
//   3D  Ex: (Ex[i,j] + Ex[i+1,j])/2, Ey: (Ey[i,j] + Ey[i,j+1])/2,
//       Hx, Hy: 4-point averages over (j or i) x (kc, kc+1).
// ---------------------------------------------------------------------------
template <typename T> struct FoldParams {
  int mode, nx, ny, nf, nt, nslot, ncomp;
  long long plane;
  const T *ring;
  double2 *acc;
  const double *tw[4];  // cosE sinE cosH sinH
  int wlo0, whi0, wlo1, whi1;
  const int *state;
};

template <typename T, bool EXACT>
__device__ __forceinline__ double coloc(const FoldParams<T> &fp, int port, int comp, int s, int i, int j) {
  using A = Ar<double, EXACT>;
  const T *r = fp.ring + ((long long)s * 2 + port) * fp.nslot * fp.plane;
  const long long P = fp.plane;
  if (fp.mode == OIDT_MODE_TM2) {
    if (comp == 0) return (double)r[j];
    return A::mul(0.5, A::add((double)r[P + j], (double)r[2 * P + j]));
  }
  if (fp.mode == OIDT_MODE_TE2) {
    if (comp == 0) return A::mul(0.5, A::add((double)r[j], (double)r[j + 1]));
    double a = A::add(A::add(A::add((double)r[P + j], (double)r[2 * P + j]), (double)r[P + j + 1]),
                      (double)r[2 * P + j + 1]);
    return A::mul(0.25, a);
  }
  const long long c = (long long)i * fp.ny + j;
  switch (comp) {
    case 0: return A::mul(0.5, A::add((double)r[c], (double)r[c + fp.ny]));
    case 1: return A::mul(0.5, A::add((double)r[P + c], (double)r[P + c + 1]));
    case 2: {
      double a = A::add(A::add(A::add((double)r[2 * P + c], (double)r[2 * P + c + 1]), (double)r[3 * P + c]),
                        (double)r[3 * P + c + 1]);
      return A::mul(0.25, a);
    }
    default: {
      double a = A::add(A::add(A::add((double)r[4 * P + c], (double)r[4 * P + c + fp.ny]), (double)r[5 * P + c]),
                        (double)r[5 * P + c + fp.ny]);
      return A::mul(0.25, a);
    }
  }
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_fold(FoldParams<T> fp, int count) {
  using A = Ar<double, EXACT>;
  const int wj = fp.whi1 - fp.wlo1;
  const int wi = fp.mode == OIDT_MODE_YEE3D ? fp.whi0 - fp.wlo0 : 1;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= wi * wj) return;
  const int i = fp.mode == OIDT_MODE_YEE3D ? fp.wlo0 + w / wj : 0;
  const int j = fp.wlo1 + w % wj;
  const int port = blockIdx.z / fp.ncomp, comp = blockIdx.z % fp.ncomp;
  const bool hcomp = fp.mode == OIDT_MODE_YEE3D ? comp >= 2 : comp == 1;
  const double *cs = fp.tw[hcomp ? 2 : 0], *sn = fp.tw[hcomp ? 3 : 1];
  const int f0 = blockIdx.y * kFoldF;
  const int nfc = min(kFoldF, fp.nf - f0);
  const long long cell = fp.mode == OIDT_MODE_YEE3D ? (long long)i * fp.ny + j : j;
  double2 *acc = fp.acc + (((long long)port * fp.ncomp + comp) * fp.nf + f0) * fp.plane + cell;
  double re[kFoldF], im[kFoldF];
#pragma unroll
  for (int f = 0; f < kFoldF; ++f)
    if (f < nfc) { double2 a = acc[f * fp.plane]; re[f] = a.x; im[f] = a.y; }
  const int n0 = fp.state[0];
  for (int s = 0; s < count; ++s) {
    const double x = coloc<T, EXACT>(fp, port, comp, s, i, j);
    const long long n = n0 + s;
#pragma unroll
    for (int f = 0; f < kFoldF; ++f) {
      if (f < nfc) {
        const long long t = (long long)(f0 + f) * fp.nt + n;
        re[f] = A::add(re[f], A::mul(x, __ldg(cs + t)));
        im[f] = A::sub(im[f], A::mul(x, __ldg(sn + t)));
      }
    }
  }
#pragma unroll
  for (int f = 0; f < kFoldF; ++f)
    if (f < nfc) acc[f * fp.plane] = make_double2(re[f], im[f]);
}

__global__ void k_bump(int *state, int count) {
  if (threadIdx.x == 0 && blockIdx.x == 0) state[0] += count;
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes);
    return o;
  }
};

int ncomp_of(int mode) { return mode == OIDT_MODE_YEE3D ? 4 : 2; }
int nslot_of(int mode) { return mode == OIDT_MODE_YEE3D ? 6 : 3; }

// (field, slab axis) pairs with CPML psi arrays per solver, in the reference's
// PSI_<F>_<A> naming.
std::vector<std::pair<int, int>> psi_pairs(int mode) {
  if (mode == OIDT_MODE_TM2) return {{EZ, AX}, {EZ, AY}, {HX, AY}, {HY, AX}};
  if (mode == OIDT_MODE_TE2) return {{EX, AY}, {EY, AX}, {HZ, AX}, {HZ, AY}};
  return {{EX, AY}, {EX, AZ}, {EY, AX}, {EY, AZ}, {EZ, AX}, {EZ, AY},
          {HX, AY}, {HX, AZ}, {HY, AX}, {HY, AZ}, {HZ, AX}, {HZ, AY}};
}
std::vector<int> fields_of(int mode) {
  if (mode == OIDT_MODE_TM2) return {EZ, HX, HY};
  if (mode == OIDT_MODE_TE2) return {EX, EY, HZ};
  return {EX, EY, EZ, HX, HY, HZ};
}
std::vector<int> cb_of(int mode) {  // which cb slots are used
  if (mode == OIDT_MODE_TM2) return {2};
  if (mode == OIDT_MODE_TE2) return {0, 1};
  return {0, 1, 2};
}

long long psi_elems(int mode, int axis, int nx, int ny, int nz, int P) {
  if (mode != OIDT_MODE_YEE3D) return (long long)(axis == AX ? P * (long long)ny : (long long)nx * P);
  if (axis == AX) return (long long)P * ny * nz;
  if (axis == AY) return (long long)nx * P * nz;
  return (long long)nx * ny * P;
}

struct JobPlan {
  size_t total;
  size_t off_f[6], off_cb[3], off_kd[6], off_rkd[6], off_be, off_ce, off_bh, off_ch;
  size_t off_psi[6][3][2];
  size_t off_jsrc, off_tw[4], off_ring, off_acc, off_state, off_params;
  long long N, plane;
  int K, esz;
};

int plan_job(const oidt_job_desc *d, JobPlan *pl, std::string *why) {
  auto bad = [&](const char *m) { if (why) *why = m; return OIDT_ERR_INVALID; };
  if (!d) return bad("null descriptor");
  if (d->mode < 0 || d->mode > 2) return bad("mode must be OIDT_MODE_TM2/TE2/YEE3D");
  if (d->precision != OIDT_F32 && d->precision != OIDT_F64) return bad("precision must be OIDT_F32 or OIDT_F64");
  if (d->arith != OIDT_ARITH_FAST && d->arith != OIDT_ARITH_EXACT) return bad("arith must be FAST or EXACT");
  const bool is3 = d->mode == OIDT_MODE_YEE3D;
  if (d->nx < 5 || d->ny < 5 || (is3 ? d->nz < 5 : d->nz != 1)) return bad("grid too small (or nz != 1 in 2D)");
  const int P = d->num_cpml;
  if (P < 1) return bad("num_cpml must be >= 1");
  if (d->ib < 1 || d->jb < 1 || (is3 && d->kb < 1)) return bad("update limits ib/jb/kb must be >= 1");
  if (d->ie > d->nx - 1 || d->je > d->ny - 1 || (is3 && d->ke > d->nz - 1))
    return bad("update limits ie/je/ke must leave one ghost cell");
  // Low and high CPML slabs must not share cells (the reference's psi kernels
  // would race on such grids).
  if (d->ie - d->ib < 2 * P || d->je - d->jb < 2 * P || (is3 && d->ke - d->kb < 2 * P))
    return bad("domain narrower than two CPML slabs");
  if (d->nt < 1 || d->nf < 1) return bad("nt and nf must be >= 1");
  if (!d->j_src || !d->cos_e || !d->sin_e || !d->cos_h || !d->sin_h || !d->be || !d->ce || !d->bh || !d->ch)
    return bad("missing source, twiddle or CPML arrays");
  for (int c : cb_of(d->mode))
    if (!d->cb[c]) return bad("missing cb array");
  for (int a = 0; a < 6; ++a)
    if (!d->kdx[a] && (is3 || (a != 2 && a != 5))) return bad("missing kappa*dx array");
  const int along = is3 ? 2 : 0;  // port planes: z (3D) or x (2D)
  const int nalong = is3 ? d->nz : d->nx;
  for (int q = 0; q < 2; ++q)
    if (d->port_pos[q] < 0 || d->port_pos[q] + 1 >= nalong) return bad("port plane out of range");
  (void)along;
  if (d->win_lo[1] < 0 || d->win_hi[1] > d->ny - 1 || d->win_lo[1] >= d->win_hi[1]) return bad("bad DFT window (j)");
  if (is3 && (d->win_lo[0] < 0 || d->win_hi[0] > d->nx - 1 || d->win_lo[0] >= d->win_hi[0]))
    return bad("bad DFT window (i)");
  if (d->src_field >= 0) {
    const std::vector<int> fl = fields_of(d->mode);
    if (std::find(fl.begin(), fl.end(), d->src_field) == fl.end()) return bad("source field not in this solver");
    const int lim_lo[3] = {d->ib, d->jb, is3 ? d->kb : 0};
    const int lim_hi[3] = {d->ie, d->je, is3 ? d->ke : 1};
    for (int a = 0; a < (is3 ? 3 : 2); ++a) {
      if (d->src_lo[a] > d->src_hi[a]) return bad("source box inverted");
      if (d->src_lo[a] < d->src_hi[a] && (d->src_lo[a] <= lim_lo[a] || d->src_hi[a] > lim_hi[a]))
        return bad("source box must lie inside the updated interior");
    }
  }
  const int esz = d->precision == OIDT_F32 ? 4 : 8;
  const long long N = (long long)d->nx * d->ny * d->nz;
  const long long plane = is3 ? (long long)d->nx * d->ny : d->ny;
  const int K = d->ring_steps > 0 ? d->ring_steps : kDefaultRing;
  if (K > 4096) return bad("ring_steps too large");
  Layout L;
  memset(pl, 0, sizeof(*pl));
  for (int f : fields_of(d->mode)) pl->off_f[f] = L.take(N * esz);
  for (int c : cb_of(d->mode)) pl->off_cb[c] = L.take(N * esz);
  const int dims[3] = {d->nx, d->ny, d->nz};
  for (int a = 0; a < 6; ++a) {
    if (!is3 && (a == 2 || a == 5)) continue;
    pl->off_kd[a] = L.take((size_t)dims[a % 3] * esz);
    pl->off_rkd[a] = L.take((size_t)dims[a % 3] * esz);
  }
  pl->off_be = L.take(P * esz);
  pl->off_ce = L.take(P * esz);
  pl->off_bh = L.take(P * esz);
  pl->off_ch = L.take(P * esz);
  for (auto fa : psi_pairs(d->mode))
    for (int sd = 0; sd < 2; ++sd)
      pl->off_psi[fa.first][fa.second][sd] = L.take(psi_elems(d->mode, fa.second, d->nx, d->ny, d->nz, P) * esz);
  pl->off_jsrc = L.take((size_t)d->nt * esz);
  for (int t = 0; t < 4; ++t) pl->off_tw[t] = L.take((size_t)d->nf * d->nt * 8);
  pl->off_ring = L.take((size_t)K * 2 * nslot_of(d->mode) * plane * esz);
  pl->off_acc = L.take((size_t)2 * ncomp_of(d->mode) * d->nf * plane * 16);
  pl->off_state = L.take(64);
  pl->off_params = L.take(std::max(sizeof(Params<float>), sizeof(Params<double>)));
  pl->total = L.off;
  pl->N = N;
  pl->plane = plane;
  pl->K = K;
  pl->esz = esz;
  return OIDT_OK;
}

struct Job {
  uint64_t id = 0;
  oidt_job_desc d{};
  JobPlan pl{};
  unsigned char *mem = nullptr;
  Params<float> pf{};
  Params<double> pd{};
  FoldParams<float> ff{};
  FoldParams<double> fd{};
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ready = nullptr;  // uploads finished
  cudaEvent_t done = nullptr;   // last enqueued work finished
  long long steps_enqueued = 0;
  bool busy = false;
};

struct BatchPlan {  // cached multi-job composition
  std::vector<uint64_t> ids;
  Tile *tiles = nullptr;
  int ntiles = 0;
  cudaGraphExec_t graph = nullptr;
  int K = 0;
};

}  // namespace

struct oidt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;  // compute
  cudaStream_t upload = nullptr;  // job creation copies
  uint64_t budget = 0, in_use = 0;
  std::map<uint64_t, Job *> jobs;
  uint64_t next_id = 1;
  std::mutex mu;
  std::string err;
  long long launches = 0;
  BatchPlan batch;
};

namespace {

int fail(oidt_ctx *ctx, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return code;
}

#define CU(ctx, call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(ctx, OIDT_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <typename T> Params<T> &params_of(Job *j);
template <> Params<float> &params_of<float>(Job *j) { return j->pf; }
template <> Params<double> &params_of<double>(Job *j) { return j->pd; }
template <typename T> FoldParams<T> &fold_of(Job *j);
template <> FoldParams<float> &fold_of<float>(Job *j) { return j->ff; }
template <> FoldParams<double> &fold_of<double>(Job *j) { return j->fd; }

template <typename T> void fill_params(Job *J) {
  const oidt_job_desc &d = J->d;
  const JobPlan &pl = J->pl;
  unsigned char *m = J->mem;
  Params<T> &p = params_of<T>(J);
  memset(&p, 0, sizeof p);
  p.mode = d.mode;
  p.nx = d.nx; p.ny = d.ny; p.nz = d.nz;
  p.P = d.num_cpml;
  p.ib = d.ib; p.jb = d.jb; p.kb = d.kb; p.ie = d.ie; p.je = d.je; p.ke = d.ke;
  for (int f : fields_of(d.mode)) p.f[f] = reinterpret_cast<T *>(m + pl.off_f[f]);
  for (int c : cb_of(d.mode)) p.cb[c] = reinterpret_cast<const T *>(m + pl.off_cb[c]);
  for (int a = 0; a < 6; ++a) {
    if (d.mode != OIDT_MODE_YEE3D && (a == 2 || a == 5)) continue;
    p.kd[a] = reinterpret_cast<const T *>(m + pl.off_kd[a]);
    p.rkd[a] = reinterpret_cast<const T *>(m + pl.off_rkd[a]);
  }
  p.be = reinterpret_cast<const T *>(m + pl.off_be);
  p.ce = reinterpret_cast<const T *>(m + pl.off_ce);
  p.bh = reinterpret_cast<const T *>(m + pl.off_bh);
  p.ch = reinterpret_cast<const T *>(m + pl.off_ch);
  p.db = (T)d.db;
  p.dx = (T)d.dx;
  p.rdx = (T)(1.0 / (double)p.dx);
  for (auto fa : psi_pairs(d.mode))
    for (int sd = 0; sd < 2; ++sd) p.psi[fa.first][fa.second][sd] = reinterpret_cast<T *>(m + pl.off_psi[fa.first][fa.second][sd]);
  p.src_field = d.src_field;
  for (int a = 0; a < 3; ++a) { p.slo[a] = d.src_lo[a]; p.shi[a] = d.src_hi[a]; }
  if (d.mode != OIDT_MODE_YEE3D) { p.slo[2] = 0; p.shi[2] = 1; }
  p.jsrc = reinterpret_cast<const T *>(m + pl.off_jsrc);
  p.ring = reinterpret_cast<T *>(m + pl.off_ring);
  p.ring_K = pl.K;
  p.nslot = nslot_of(d.mode);
  p.plane = pl.plane;
  p.port_pos[0] = d.port_pos[0];
  p.port_pos[1] = d.port_pos[1];
  p.state = reinterpret_cast<int *>(m + pl.off_state);

  FoldParams<T> &fp = fold_of<T>(J);
  memset(&fp, 0, sizeof fp);
  fp.mode = d.mode; fp.nx = d.nx; fp.ny = d.ny; fp.nf = d.nf; fp.nt = d.nt;
  fp.nslot = nslot_of(d.mode); fp.ncomp = ncomp_of(d.mode); fp.plane = pl.plane;
  fp.ring = p.ring;
  fp.acc = reinterpret_cast<double2 *>(m + pl.off_acc);
  for (int t = 0; t < 4; ++t) fp.tw[t] = reinterpret_cast<const double *>(m + pl.off_tw[t]);
  fp.wlo0 = d.win_lo[0]; fp.whi0 = d.win_hi[0]; fp.wlo1 = d.win_lo[1]; fp.whi1 = d.win_hi[1];
  fp.state = p.state;
}

template <typename T> int upload(oidt_ctx *ctx, Job *J, const oidt_job_desc *src) {
  const oidt_job_desc &d = *src;
  const JobPlan &pl = J->pl;
  unsigned char *m = J->mem;
  cudaStream_t st = ctx->upload;
  CU(ctx, cudaMemsetAsync(m, 0, pl.total, st));
  const size_t N = pl.N * sizeof(T);
  for (int c : cb_of(d.mode)) CU(ctx, cudaMemcpyAsync(m + pl.off_cb[c], d.cb[c], N, cudaMemcpyHostToDevice, st));
  const int dims[3] = {d.nx, d.ny, d.nz};
  std::vector<T> rk;
  for (int a = 0; a < 6; ++a) {
    if (d.mode != OIDT_MODE_YEE3D && (a == 2 || a == 5)) continue;
    const int n = dims[a % 3];
    const T *kd = static_cast<const T *>(d.kdx[a]);
    CU(ctx, cudaMemcpyAsync(m + pl.off_kd[a], kd, n * sizeof(T), cudaMemcpyHostToDevice, st));
    rk.resize(n);
    for (int i = 0; i < n; ++i) rk[i] = (T)1 / kd[i];
    CU(ctx, cudaMemcpyAsync(m + pl.off_rkd[a], rk.data(), n * sizeof(T), cudaMemcpyHostToDevice, st));
    CU(ctx, cudaStreamSynchronize(st));  // rk is reused
  }
  const int P = d.num_cpml;
  CU(ctx, cudaMemcpyAsync(m + pl.off_be, d.be, P * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(ctx, cudaMemcpyAsync(m + pl.off_ce, d.ce, P * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(ctx, cudaMemcpyAsync(m + pl.off_bh, d.bh, P * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(ctx, cudaMemcpyAsync(m + pl.off_ch, d.ch, P * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(ctx, cudaMemcpyAsync(m + pl.off_jsrc, d.j_src, d.nt * sizeof(T), cudaMemcpyHostToDevice, st));
  const double *tw[4] = {d.cos_e, d.sin_e, d.cos_h, d.sin_h};
  for (int t = 0; t < 4; ++t)
    CU(ctx, cudaMemcpyAsync(m + pl.off_tw[t], tw[t], (size_t)d.nf * d.nt * 8, cudaMemcpyHostToDevice, st));
  fill_params<T>(J);
  CU(ctx, cudaMemcpyAsync(m + pl.off_params, &params_of<T>(J), sizeof(Params<T>), cudaMemcpyHostToDevice, st));
  CU(ctx, cudaEventRecord(J->ready, st));
  // Host buffers are borrowed only for this call.
  CU(ctx, cudaStreamSynchronize(st));
  return OIDT_OK;
}

template <typename T, bool EXACT> void launch_step(oidt_ctx *ctx, Job *J, int s, cudaStream_t st) {
  Params<T> &p = params_of<T>(J);
  if (J->d.mode == OIDT_MODE_YEE3D) {
    dim3 blk(kBlock3Z, kBlock3Y), grd((p.nz + kBlock3Z - 1) / kBlock3Z, (p.ny + kBlock3Y - 1) / kBlock3Y, p.nx);
    k_y3_e<T, EXACT><<<grd, blk, 0, st>>>(p, s);
    k_y3_h<T, EXACT><<<grd, blk, 0, st>>>(p, s);
  } else {
    dim3 blk(kBlock2), grd((p.ny + kBlock2 - 1) / kBlock2, p.nx);
    k_2d_e<T, EXACT><<<grd, blk, 0, st>>>(p, s);
    k_2d_h<T, EXACT><<<grd, blk, 0, st>>>(p, s);
  }
  ctx->launches += 2;
}

template <typename T, bool EXACT> void launch_fold(oidt_ctx *ctx, Job *J, int count, cudaStream_t st) {
  FoldParams<T> &fp = fold_of<T>(J);
  const int wj = fp.whi1 - fp.wlo1;
  const int wi = J->d.mode == OIDT_MODE_YEE3D ? fp.whi0 - fp.wlo0 : 1;
  dim3 grd((wi * wj + 127) / 128, (fp.nf + kFoldF - 1) / kFoldF, 2 * fp.ncomp);
  k_fold<T, EXACT><<<grd, 128, 0, st>>>(fp, count);
  k_bump<<<1, 32, 0, st>>>(params_of<T>(J).state, count);
  ctx->launches += 2;
}

template <typename T, bool EXACT> int advance_t(oidt_ctx *ctx, Job *J, int nsteps) {
  cudaStream_t st = ctx->stream;
  CU(ctx, cudaStreamWaitEvent(st, J->ready, 0));
  const int K = J->pl.K;
  int left = nsteps;
  while (left > 0) {
    const int cnt = std::min(K, left);
    if (cnt == K) {
      if (!J->graph) {
        cudaGraph_t g;
        CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        long long before = ctx->launches;
        for (int s = 0; s < K; ++s) launch_step<T, EXACT>(ctx, J, s, st);
        launch_fold<T, EXACT>(ctx, J, K, st);
        ctx->launches = before;  // counted at replay
        CU(ctx, cudaStreamEndCapture(st, &g));
        CU(ctx, cudaGraphInstantiate(&J->graph, g, 0));
        CU(ctx, cudaGraphDestroy(g));
      }
      CU(ctx, cudaGraphLaunch(J->graph, st));
      ctx->launches += 2 * K + 2;
    } else {
      for (int s = 0; s < cnt; ++s) launch_step<T, EXACT>(ctx, J, s, st);
      launch_fold<T, EXACT>(ctx, J, cnt, st);
    }
    left -= cnt;
  }
  CU(ctx, cudaGetLastError());
  J->steps_enqueued += nsteps;
  CU(ctx, cudaEventRecord(J->done, st));
  J->busy = true;
  return OIDT_OK;
}

int advance(oidt_ctx *ctx, Job *J, int nsteps) {
  const bool f64 = J->d.precision == OIDT_F64, ex = J->d.arith == OIDT_ARITH_EXACT;
  if (f64) return ex ? advance_t<double, true>(ctx, J, nsteps) : advance_t<double, false>(ctx, J, nsteps);
  return ex ? advance_t<float, true>(ctx, J, nsteps) : advance_t<float, false>(ctx, J, nsteps);
}

// ---- multi-job launches ----------------------------------------------------
std::vector<Tile> make_tiles(const std::vector<Job *> &js) {
  std::vector<Tile> t;
  for (int b = 0; b < (int)js.size(); ++b) {
    const oidt_job_desc &d = js[b]->d;
    if (d.mode == OIDT_MODE_YEE3D) {
      for (int i = 0; i < d.nx; ++i)
        for (int j0 = 0; j0 < d.ny; j0 += kBlock3Y)
          for (int k0 = 0; k0 < d.nz; k0 += kBlock3Z) t.push_back({b, i, j0, k0});
    } else {
      for (int i = 0; i < d.nx; ++i)
        for (int j0 = 0; j0 < d.ny; j0 += kBlock2) t.push_back({b, i, j0, 0});
    }
  }
  return t;
}

template <typename T, bool EXACT>
int batch_t(oidt_ctx *ctx, std::vector<Job *> &js, int nsteps) {
  cudaStream_t st = ctx->stream;
  BatchPlan &bp = ctx->batch;
  std::vector<uint64_t> ids;
  for (Job *j : js) ids.push_back(j->id);
  const int K = js[0]->pl.K;
  for (Job *j : js) {
    if (j->pl.K != K) return fail(ctx, OIDT_ERR_INVALID, "batched jobs must share ring_steps");
    CU(ctx, cudaStreamWaitEvent(st, j->ready, 0));
  }
  if (bp.ids != ids || bp.K != K) {
    if (bp.graph) { cudaGraphExecDestroy(bp.graph); bp.graph = nullptr; }
    if (bp.tiles) { cudaFree(bp.tiles); bp.tiles = nullptr; }
    std::vector<Tile> t = make_tiles(js);
    // Params of job b must sit at params[b]: gather them into one array.
    CU(ctx, cudaMalloc(&bp.tiles, t.size() * sizeof(Tile) + js.size() * sizeof(Params<T>) + 256));
    CU(ctx, cudaMemcpy(bp.tiles, t.data(), t.size() * sizeof(Tile), cudaMemcpyHostToDevice));
    Params<T> *dp = reinterpret_cast<Params<T> *>(reinterpret_cast<unsigned char *>(bp.tiles) +
                                                  align_up(t.size() * sizeof(Tile)));
    std::vector<Params<T>> hp;
    for (Job *j : js) hp.push_back(params_of<T>(j));
    CU(ctx, cudaMemcpy(dp, hp.data(), hp.size() * sizeof(Params<T>), cudaMemcpyHostToDevice));
    bp.ntiles = (int)t.size();
    bp.ids = ids;
    bp.K = K;
  }
  const Params<T> *dp = reinterpret_cast<const Params<T> *>(reinterpret_cast<unsigned char *>(bp.tiles) +
                                                            align_up(bp.ntiles * sizeof(Tile)));
  auto block = [&](int cnt) {
    for (int s = 0; s < cnt; ++s) {
      k_batch<T, EXACT, true><<<bp.ntiles, 128, 0, st>>>(dp, bp.tiles, s);
      k_batch<T, EXACT, false><<<bp.ntiles, 128, 0, st>>>(dp, bp.tiles, s);
    }
    for (Job *j : js) launch_fold<T, EXACT>(ctx, j, cnt, st);
    ctx->launches += 2 * cnt;
  };
  int left = nsteps;
  while (left > 0) {
    const int cnt = std::min(K, left);
    if (cnt == K) {
      if (!bp.graph) {
        cudaGraph_t g;
        long long before = ctx->launches;
        CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        block(K);
        CU(ctx, cudaStreamEndCapture(st, &g));
        ctx->launches = before;
        CU(ctx, cudaGraphInstantiate(&bp.graph, g, 0));
        CU(ctx, cudaGraphDestroy(g));
      }
      CU(ctx, cudaGraphLaunch(bp.graph, st));
      ctx->launches += 2 * K + 2 * (long long)js.size();
    } else {
      block(cnt);
    }
    left -= cnt;
  }
  CU(ctx, cudaGetLastError());
  for (Job *j : js) {
    j->steps_enqueued += nsteps;
    CU(ctx, cudaEventRecord(j->done, st));
    j->busy = true;
  }
  return OIDT_OK;
}

Job *find(oidt_ctx *ctx, uint64_t id) {
  auto it = ctx->jobs.find(id);
  return it == ctx->jobs.end() ? nullptr : it->second;
}

int wait_event(oidt_ctx *ctx, cudaEvent_t ev, int timeout_ms) {
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return OIDT_OK;
    if (e != cudaErrorNotReady) return fail(ctx, OIDT_ERR_CUDA, "device error: %s", cudaGetErrorString(e));
    if (timeout_ms >= 0) {
      auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
      if (ms >= timeout_ms) return fail(ctx, OIDT_ERR_TIMEOUT, "wait timed out after %d ms", timeout_ms);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int32_t oidt_abi_version(void) { return OIDT_ABI_VERSION; }

int32_t oidt_create(int32_t device, uint64_t hbm_budget, oidt_ctx **out) {
  if (!out) return OIDT_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return OIDT_ERR_CUDA;
  oidt_ctx *ctx = new oidt_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return OIDT_ERR_CUDA;
  }
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  ctx->budget = hbm_budget ? hbm_budget : (uint64_t)(0.9 * (double)fr);
  *out = ctx;
  return OIDT_OK;
}

int32_t oidt_destroy(oidt_ctx *ctx) {
  if (!ctx) return OIDT_ERR_INVALID;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &kv : ctx->jobs) {
      Job *J = kv.second;
      if (J->graph) cudaGraphExecDestroy(J->graph);
      cudaFreeAsync(J->mem, ctx->stream);
      cudaEventDestroy(J->ready);
      cudaEventDestroy(J->done);
      delete J;
    }
    ctx->jobs.clear();
    if (ctx->batch.graph) cudaGraphExecDestroy(ctx->batch.graph);
    if (ctx->batch.tiles) cudaFree(ctx->batch.tiles);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    cudaStreamDestroy(ctx->upload);
  }
  delete ctx;
  return OIDT_OK;
}

const char *oidt_last_error(oidt_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int32_t oidt_stats_get(oidt_ctx *ctx, oidt_stats *out) {
  if (!ctx || !out) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  out->hbm_budget = ctx->budget;
  out->hbm_in_use = ctx->in_use;
  out->live_jobs = (int32_t)ctx->jobs.size();
  out->device = ctx->device;
  out->kernel_launches = ctx->launches;
  return OIDT_OK;
}

int32_t oidt_job_bytes(const oidt_job_desc *desc, uint64_t *bytes) {
  JobPlan pl;
  int rc = plan_job(desc, &pl, nullptr);
  if (rc) return rc;
  if (bytes) *bytes = pl.total;
  return OIDT_OK;
}

int32_t oidt_job_create(oidt_ctx *ctx, const oidt_job_desc *desc, uint64_t *job) {
  if (!ctx || !job) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  JobPlan pl;
  std::string why;
  int rc = plan_job(desc, &pl, &why);
  if (rc) return fail(ctx, rc, "invalid job: %s", why.c_str());
  if (ctx->in_use + pl.total > ctx->budget)
    return fail(ctx, OIDT_ERR_BUDGET, "job needs %llu bytes; %llu of %llu in use", (unsigned long long)pl.total,
                (unsigned long long)ctx->in_use, (unsigned long long)ctx->budget);
  CU(ctx, cudaSetDevice(ctx->device));
  Job *J = new Job();
  J->d = *desc;
  J->pl = pl;
  if (cudaMallocAsync(reinterpret_cast<void **>(&J->mem), pl.total, ctx->upload) != cudaSuccess) {
    delete J;
    cudaGetLastError();
    return fail(ctx, OIDT_ERR_BUDGET, "device allocation of %llu bytes failed", (unsigned long long)pl.total);
  }
  cudaEventCreateWithFlags(&J->ready, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&J->done, cudaEventDisableTiming);
  rc = desc->precision == OIDT_F64 ? upload<double>(ctx, J, desc) : upload<float>(ctx, J, desc);
  if (rc) {
    cudaFreeAsync(J->mem, ctx->upload);
    cudaStreamSynchronize(ctx->upload);
    cudaEventDestroy(J->ready);
    cudaEventDestroy(J->done);
    delete J;
    return rc;
  }
  // Host pointers are not kept.
  memset(J->d.cb, 0, sizeof J->d.cb);
  memset(J->d.kdx, 0, sizeof J->d.kdx);
  J->d.be = J->d.ce = J->d.bh = J->d.ch = J->d.j_src = nullptr;
  J->d.cos_e = J->d.sin_e = J->d.cos_h = J->d.sin_h = nullptr;
  J->id = ctx->next_id++;
  ctx->jobs[J->id] = J;
  ctx->in_use += pl.total;
  *job = J->id;
  return OIDT_OK;
}

int32_t oidt_job_advance(oidt_ctx *ctx, uint64_t job, int32_t nsteps) {
  if (!ctx) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  if (nsteps < 0) return fail(ctx, OIDT_ERR_INVALID, "nsteps < 0");
  if (J->steps_enqueued + nsteps > J->d.nt)
    return fail(ctx, OIDT_ERR_STATE, "job has %d source steps; %lld done, %d more requested", J->d.nt,
                J->steps_enqueued, nsteps);
  if (nsteps == 0) return OIDT_OK;
  CU(ctx, cudaSetDevice(ctx->device));
  return advance(ctx, J, nsteps);
}

int32_t oidt_batch_advance(oidt_ctx *ctx, const uint64_t *jobs, int32_t njobs, int32_t nsteps) {
  if (!ctx || !jobs || njobs <= 0 || nsteps < 0) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  std::vector<Job *> js;
  for (int b = 0; b < njobs; ++b) {
    Job *J = find(ctx, jobs[b]);
    if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)jobs[b]);
    if (J->steps_enqueued + nsteps > J->d.nt) return fail(ctx, OIDT_ERR_STATE, "job %llu has too few source steps", (unsigned long long)jobs[b]);
    if (!js.empty() && (J->d.precision != js[0]->d.precision || J->d.arith != js[0]->d.arith))
      return fail(ctx, OIDT_ERR_INVALID, "batched jobs must share precision and arithmetic");
    js.push_back(J);
  }
  if (nsteps == 0) return OIDT_OK;
  CU(ctx, cudaSetDevice(ctx->device));
  const bool f64 = js[0]->d.precision == OIDT_F64, ex = js[0]->d.arith == OIDT_ARITH_EXACT;
  if (f64) return ex ? batch_t<double, true>(ctx, js, nsteps) : batch_t<double, false>(ctx, js, nsteps);
  return ex ? batch_t<float, true>(ctx, js, nsteps) : batch_t<float, false>(ctx, js, nsteps);
}

int32_t oidt_job_sync(oidt_ctx *ctx, uint64_t job, int32_t timeout_ms) {
  if (!ctx) return OIDT_ERR_INVALID;
  cudaEvent_t ev;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    Job *J = find(ctx, job);
    if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
    if (!J->busy) return OIDT_OK;
    ev = J->done;
  }
  cudaSetDevice(ctx->device);
  int rc = wait_event(ctx, ev, timeout_ms);
  if (rc == OIDT_OK) {
    std::lock_guard<std::mutex> g(ctx->mu);
    Job *J = find(ctx, job);
    if (J && J->done == ev) J->busy = cudaEventQuery(ev) != cudaSuccess;
  }
  return rc;
}

int32_t oidt_job_query(oidt_ctx *ctx, uint64_t job, int32_t *steps_done, int32_t *busy) {
  if (!ctx) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  cudaSetDevice(ctx->device);
  const bool b = J->busy && cudaEventQuery(J->done) == cudaErrorNotReady;
  if (!b) J->busy = false;
  if (busy) *busy = b ? 1 : 0;
  if (steps_done) *steps_done = b ? -1 : (int32_t)J->steps_enqueued;
  return OIDT_OK;
}

static int read_common(oidt_ctx *ctx, Job *J) {
  CU(ctx, cudaSetDevice(ctx->device));
  CU(ctx, cudaEventSynchronize(J->done));
  CU(ctx, cudaStreamSynchronize(ctx->upload));
  return OIDT_OK;
}

int32_t oidt_job_read_dft(oidt_ctx *ctx, uint64_t job, int32_t port, int32_t comp, double *out, size_t n) {
  if (!ctx || !out) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  const int nc = ncomp_of(J->d.mode);
  if (port < 0 || port > 1 || comp < 0 || comp >= nc) return fail(ctx, OIDT_ERR_INVALID, "bad port/comp");
  const size_t need = (size_t)2 * J->d.nf * J->pl.plane;
  if (n < need) return fail(ctx, OIDT_ERR_INVALID, "output needs %zu doubles", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  const unsigned char *src = J->mem + J->pl.off_acc + ((size_t)port * nc + comp) * J->d.nf * J->pl.plane * 16;
  CU(ctx, cudaMemcpy(out, src, need * 8, cudaMemcpyDeviceToHost));
  return OIDT_OK;
}

static bool field_ok(Job *J, int field) {
  if (field < 0 || field > 5) return false;
  std::vector<int> f = fields_of(J->d.mode);
  return std::find(f.begin(), f.end(), field) != f.end();
}

int32_t oidt_job_read_field(oidt_ctx *ctx, uint64_t job, int32_t field, void *out, size_t nbytes) {
  if (!ctx || !out) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  if (!field_ok(J, field)) return fail(ctx, OIDT_ERR_INVALID, "field %d not in this solver", field);
  const size_t need = J->pl.N * J->pl.esz;
  if (nbytes < need) return fail(ctx, OIDT_ERR_INVALID, "output needs %zu bytes", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  CU(ctx, cudaMemcpy(out, J->mem + J->pl.off_f[field], need, cudaMemcpyDeviceToHost));
  return OIDT_OK;
}

int32_t oidt_job_write_field(oidt_ctx *ctx, uint64_t job, int32_t field, const void *src, size_t nbytes) {
  if (!ctx || !src) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  if (!field_ok(J, field)) return fail(ctx, OIDT_ERR_INVALID, "field %d not in this solver", field);
  const size_t need = J->pl.N * J->pl.esz;
  if (nbytes != need) return fail(ctx, OIDT_ERR_INVALID, "input must be %zu bytes", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  CU(ctx, cudaMemcpy(J->mem + J->pl.off_f[field], src, need, cudaMemcpyHostToDevice));
  return OIDT_OK;
}

int32_t oidt_job_read_psi(oidt_ctx *ctx, uint64_t job, int32_t field, int32_t axis, int32_t side, void *out,
                          size_t nbytes) {
  if (!ctx || !out) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  bool ok = false;
  for (auto fa : psi_pairs(J->d.mode)) ok |= (fa.first == field && fa.second == axis);
  if (!ok || side < 0 || side > 1) return fail(ctx, OIDT_ERR_INVALID, "no psi array for field %d axis %d", field, axis);
  const size_t need = psi_elems(J->d.mode, axis, J->d.nx, J->d.ny, J->d.nz, J->d.num_cpml) * J->pl.esz;
  if (nbytes < need) return fail(ctx, OIDT_ERR_INVALID, "output needs %zu bytes", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  CU(ctx, cudaMemcpy(out, J->mem + J->pl.off_psi[field][axis][side], need, cudaMemcpyDeviceToHost));
  return OIDT_OK;
}

int32_t oidt_job_release(oidt_ctx *ctx, uint64_t job) {
  if (!ctx) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  CU(ctx, cudaSetDevice(ctx->device));
  CU(ctx, cudaEventSynchronize(J->done));
  if (J->graph) cudaGraphExecDestroy(J->graph);
  if (std::find(ctx->batch.ids.begin(), ctx->batch.ids.end(), job) != ctx->batch.ids.end()) {
    if (ctx->batch.graph) cudaGraphExecDestroy(ctx->batch.graph);
    ctx->batch.graph = nullptr;
    ctx->batch.ids.clear();
  }
  cudaFreeAsync(J->mem, ctx->stream);  // stream-ordered: no device-wide synchronisation
  cudaEventDestroy(J->ready);
  cudaEventDestroy(J->done);
  ctx->in_use -= J->pl.total;
  ctx->jobs.erase(job);
  delete J;
  return OIDT_OK;
}

}  // extern "C"
