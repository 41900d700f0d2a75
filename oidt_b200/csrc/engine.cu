// engine.cu -- liboidt.so: job management, launches and the C ABI (include/oidt.h).
//
// Device layout of one job (one cudaMallocAsync block, 256-byte aligned
// sub-buffers): fields and dt/eps grids in the reference layout ([nx][ny] or
// [nx][ny][nz], C order; 3D rows along z padded to a multiple of 4 cells so
// TMA row strides are 16-byte multiples), 1-D kappa*dx arrays and their
// reciprocals, CPML psi slabs in the reference's PSI_<F>_<A><LO|HI> shapes,
// the source waveform, float64 twiddle tables [nf][nt], the capture ring
// [K][port][slot][plane], float64 complex DFT accumulators
// [port][comp][nf][plane], the port-power result [nf], an optional line-probe
// record [4][nt][nx], and for the 3D plane-sweep form a second field buffer and
// a second E-psi buffer (it writes the other buffer each step).
//
// A time step is two per-cell launches (E half, H half; kernels.cuh) -- or,
// for 3D jobs that ask for it, one plane-sweep launch over the job's work
// items (sweep3d.cuh) -- then the line probe if the job has one.  Every K
// steps a fold kernel turns the captured port planes into float64 DFT updates
// and a one-thread kernel advances the step counter, so a K-step block is a
// fixed launch sequence, captured once into a CUDA graph and replayed, alone
// or as one branch of a multi-job block.  The step kernels are launched with
// programmatic stream serialization and wait for their predecessor in
// pdl_wait().  3D per-cell blocks are 32 x rows cells (rows 2, 4 or 8, a
// launch choice that leaves results unchanged).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/oidt.h"
#include "kernels.cuh"
#include "sweep3d.cuh"
#include "vec3d.cuh"
#include "tile2d.cuh"

using namespace oidt;

namespace {

constexpr int kDefaultRing = 32;
constexpr int kFoldF = 7;  // frequencies per fold thread in 3D (41 = 6 x 7 - 1); 2D: one
constexpr int kBlock3Z = 32, kRowsDefault = 4;  // 3D per-cell tile: 32 (k) x rows (j), rows 2, 4 or 8
constexpr int kBlock2 = 128;
constexpr int TY = kSweepTY, TZ = kSweepTZ, ST = kSweepStages;  // owned tile of a sweep CTA
constexpr int EYB = kSweepEY, EZB = kSweepEZ;                      // its thread box
constexpr int kVariantCell = 0, kVariantSweep = 1, kVariantVec = 2, kVariantWave = 3;  // oidt_job_desc.reserved[0]
constexpr int kVariantTile = 4;  // 2D: tiles advanced in sub-blocks of up to kTileHaloMax steps (tile2d.cuh)
constexpr int kTileMaxBlocks = 1024;  // tiles of a cooperative (several sub-block) launch at most
constexpr size_t kTileSmemMax = 227 * 1024;  // shared memory of a tile block at most

// ---------------------------------------------------------------------------
// Line probe (wave-impedance recording): after every step, colocated Ey, Ez,
// Hy, Hz along x at (y, z) = (jc, kc) into out[comp][n][x], x in [0, ie)
// (FDTD/GPU/FDTD_3D/wave_impedance/fdtd_funcs.py map_efield_zwave /
// map_hfield_zwave: 0.5 (a + b) and 0.25 (a + b + c + d) in that order).
// ---------------------------------------------------------------------------
template <typename T> struct ProbeArgs {
  const T *ey, *ez, *hy, *hz;  // fields holding the state after the step
  T *out;                      // [4][nt][nx]
  int nx, nt, ie, jc, kc;
  long long sy, sx;            // row and plane strides (elements)
  const int *state;            // state[0] = absolute step of ring slot 0
};

template <typename T, bool EXACT> __global__ void __launch_bounds__(128) k_probe(ProbeArgs<T> a, int s) {
  pdl_wait();
  using A = Ar<T, EXACT>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.state[0] + s;
  if (x >= a.ie || n >= a.nt) return;
  const long long c = x * a.sx + a.jc * a.sy + a.kc;  // (x, jc, kc)
  const T half = T(0.5), quarter = T(0.25);
  const size_t row = (size_t)n * a.nx + x, comp = (size_t)a.nt * a.nx;
  a.out[row] = A::mul(half, A::add(a.ey[c], a.ey[c + a.sy]));
  a.out[comp + row] = A::mul(half, A::add(a.ez[c], a.ez[c + 1]));
  a.out[2 * comp + row] =
      A::mul(quarter, A::add(A::add(A::add(a.hy[c], a.hy[c + a.sx]), a.hy[c + 1]), a.hy[c + a.sx + 1]));
  a.out[3 * comp + row] =
      A::mul(quarter, A::add(A::add(A::add(a.hz[c], a.hz[c + a.sx]), a.hz[c + a.sy]), a.hz[c + a.sx + a.sy]));
}

// ---------------------------------------------------------------------------
// Per-cell launches (2D, and the 3D per-cell variant): in place.
// ---------------------------------------------------------------------------
// A block of the 3D per-cell launches covers kBlock3Z (k) x BY (j) cells of
// one x-plane (BY = the job's tile rows: 2, 4 or 8); each warp is one (i, j) row of 32 consecutive k.  Blocks
// away from the source box run the range-masked body: the three curl
// updates, then the CPML terms -- x and y slabs uniform over the warp, z slab
// per lane -- with each component stored where its (i, j, k) range holds
// (operation order as y3_e_compute / y3_h_compute, which they equal cell by
// cell).  Blocks meeting the source box run the general per-cell code.
template <int BY, typename T>
__device__ __forceinline__ bool block_meets_src(const Params<T> &p, int i, int j0, int k0) {
  // the source box widened by one cell below in i and k (the E CPML of Ex and
  // Ez reads the Hy source at k + 1 and i + 1)
  return p.src_field >= 0 && i >= p.slo[0] - 1 && i < p.shi[0] && j0 < p.shi[1] && j0 + BY > p.slo[1] &&
         k0 < p.shi[2] && k0 + kBlock3Z > p.slo[2] - 1;
}

// Interior warps address every grid array as (per-plane base, uniform over
// the block) + (32-bit offset inside the plane), and the CPML slabs likewise;
// plan_job rejects grids whose plane or slab sizes would not fit.
template <typename T, bool EXACT, int BY>
__global__ void __launch_bounds__(32 * BY, (sizeof(T) == 4 ? 64 : 32) / BY) k_y3_e(Params<T> p, int s) {
  pdl_wait();
  const int k0 = blockIdx.x * kBlock3Z, j0 = blockIdx.y * BY, i = blockIdx.z;
  const int k = k0 + threadIdx.x, j = j0 + threadIdx.y;
  if (!block_meets_src<BY>(p, i, j0, k0)) {
    y3_e_masked<T, EXACT>(p, i, j, k, s);
    return;
  }
  if (k >= p.nz || j >= p.ny) return;
  y3_e_cell<T, EXACT>(p, i, j, k, p.state[0] + s, s);
}
template <typename T, bool EXACT, int BY>
__global__ void __launch_bounds__(32 * BY, (sizeof(T) == 4 ? 64 : 32) / BY) k_y3_h(Params<T> p, int s) {
  pdl_wait();
  // planes in decreasing i: the H half starts on the E planes the E half wrote
  // last (still in L2), and ends on the planes the next E half reads first
  const int k0 = blockIdx.x * kBlock3Z, j0 = blockIdx.y * BY, i = gridDim.z - 1 - blockIdx.z;
  const int k = k0 + threadIdx.x, j = j0 + threadIdx.y;
  if (!block_meets_src<BY>(p, i, j0, k0)) {
    y3_h_masked<T, EXACT>(p, i, j, k, s);
    return;
  }
  if (k >= p.nz || j >= p.ny) return;
  y3_h_cell<T, EXACT>(p, i, j, k, p.state[0] + s, s);
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_2d_e(Params<T> p, int s) {
  pdl_wait();
  const int j = blockIdx.x * kBlock2 + threadIdx.x, i = blockIdx.y;
  if (j >= p.ny) return;
  if (p.mode == OIDT_MODE_TM2)
    tm2_e_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
  else
    te2_e_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
}
template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_2d_h(Params<T> p, int s) {
  pdl_wait();
  // rows in decreasing i (the E half's last rows are still in L2)
  const int j = blockIdx.x * kBlock2 + threadIdx.x, i = gridDim.y - 1 - blockIdx.y;
  if (j >= p.ny) return;
  if (p.mode == OIDT_MODE_TM2)
    tm2_h_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
  else
    te2_h_cell<T, EXACT>(p, i, j, p.state[0] + s, s);
}

// ---------------------------------------------------------------------------
// DFT fold: acc[port][comp][f][cell] += sum_s x_s(cell) * (cos, -sin)[f][n0+s]
// in float64, s = 0..count-1 in order (the reference's running sum, one step
// at a time: fdtd_funcs.py simul_fft_efield/hfield).  x_s is the colocated
// port-plane sample computed from the captured raw planes:
//   TM2 E: Ez[ic,j]                   H: (Hy[ic,j] + Hy[ic+1,j]) / 2
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
  int *state;  // state[0]: absolute step of ring slot 0; state[2]: fold blocks done
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

// One block: 128 window cells x FF frequencies of one (port, component).  3D
// planes have thousands of window cells: FF = kFoldF frequencies a thread
// share each sample load; a 2D port line has a few hundred, so FF = 1 there
// (fifteen thousand short accumulation chains rather than two thousand long ones).
// The block's twiddles for up to kFoldChunk steps are staged in shared memory
// (every thread uses the same values), and so are a thread's colocated
// samples of those steps (their loads issued together rather than one ring
// latency per step); accumulators stay in registers.
constexpr int kFoldChunk = 32;
template <typename T, bool EXACT, int FF>
__global__ void __launch_bounds__(128) k_fold(FoldParams<T> fp, int count) {
  pdl_wait();
  using A = Ar<double, EXACT>;
  __shared__ double2 tw[kFoldChunk][FF];
  __shared__ double xs[kFoldChunk][128];
  const int wj = fp.whi1 - fp.wlo1;
  const int wi = fp.mode == OIDT_MODE_YEE3D ? fp.whi0 - fp.wlo0 : 1;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = w < wi * wj;
  const int i = fp.mode == OIDT_MODE_YEE3D ? fp.wlo0 + (active ? w / wj : 0) : 0;
  const int j = fp.wlo1 + (active ? w % wj : 0);
  const int port = blockIdx.z / fp.ncomp, comp = blockIdx.z % fp.ncomp;
  const bool hcomp = fp.mode == OIDT_MODE_YEE3D ? comp >= 2 : comp == 1;
  const double *cs = fp.tw[hcomp ? 2 : 0], *sn = fp.tw[hcomp ? 3 : 1];
  const int f0 = blockIdx.y * FF;
  const int nfc = min(FF, fp.nf - f0);
  const long long cell = fp.mode == OIDT_MODE_YEE3D ? (long long)i * fp.ny + j : j;
  double2 *acc = fp.acc + (((long long)port * fp.ncomp + comp) * fp.nf + f0) * fp.plane + cell;
  double re[FF], im[FF];
#pragma unroll
  for (int f = 0; f < FF; ++f) {
    re[f] = 0.0;
    im[f] = 0.0;
    if (active && f < nfc) { double2 a = acc[f * fp.plane]; re[f] = a.x; im[f] = a.y; }
  }
  const int n0 = fp.state[0];
  for (int s0 = 0; s0 < count; s0 += kFoldChunk) {
    const int sc = min(kFoldChunk, count - s0);
    __syncthreads();
    for (int t = threadIdx.x; t < sc * FF; t += blockDim.x) {
      const int ss = t / FF, f = t % FF;
      const long long idx = (long long)(f0 + f) * fp.nt + n0 + s0 + ss;
      tw[ss][f] = f < nfc ? make_double2(__ldg(cs + idx), __ldg(sn + idx)) : make_double2(0.0, 0.0);
    }
    if (active) {
#pragma unroll 8
      for (int ss = 0; ss < sc; ++ss) xs[ss][threadIdx.x] = coloc<T, EXACT>(fp, port, comp, s0 + ss, i, j);
    }
    __syncthreads();
    if (active) {
      for (int ss = 0; ss < sc; ++ss) {
        const double x = xs[ss][threadIdx.x];
#pragma unroll
        for (int f = 0; f < FF; ++f) {
          const double2 t = tw[ss][f];
          re[f] = A::add(re[f], A::mul(x, t.x));
          im[f] = A::sub(im[f], A::mul(x, t.y));
        }
      }
    }
  }
  if (active) {
#pragma unroll
    for (int f = 0; f < FF; ++f)
      if (f < nfc) acc[f * fp.plane] = make_double2(re[f], im[f]);
  }
  // the last block to finish advances the ring's step (every block has read it by then)
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    if (atomicAdd(reinterpret_cast<unsigned *>(fp.state + 2), 1u) == nb - 1) {
      fp.state[2] = 0;
      fp.state[0] += count;
    }
  }
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
bool is_e(int f) { return f <= EZ; }
// psi buffers of a field: the plane sweep double-buffers E psi (it updates H
// psi in place); the 2D tile form double-buffers every psi array.
int psi_bufs(int nbuf, int variant, int f) { return nbuf == 2 && (is_e(f) || variant == kVariantTile) ? 2 : 1; }

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

// Elements of one psi slab array in the reference's shape; `pitch` is the
// device row length along z of the x- and y-slab arrays (nz, or nzp for the
// vector form's 16-byte rows), `zpitch` that of the z-slab arrays (P, or the
// vector form's padded rows).
long long psi_elems(int mode, int axis, int nx, int ny, int nz, int P, int pitch = 0, int zpitch = 0) {
  if (mode != OIDT_MODE_YEE3D) return (long long)(axis == AX ? P * (long long)ny : (long long)nx * P);
  const long long row = pitch > 0 ? pitch : nz;
  if (axis == AX) return (long long)P * ny * row;
  if (axis == AY) return (long long)nx * P * row;
  return (long long)nx * ny * (zpitch > 0 ? zpitch : P);
}

// The vector form's z-slab psi rows.  A row holds every four-cell group that
// meets the slab: slab cell d of the low side (k = kb + d) sits at
// zoff[LO] + d = k - floor4(kb), of the high side (k = ke - P + d) at
// zoff[HI] + d = k - floor4(ke - P).  A group k0 of the slab's groups then
// reads its four values at one 16-byte aligned offset, k0 - floor4(start).
struct ZRows {
  int pitch, off[2];
};
ZRows z_rows(int kb, int ke, int P) {
  ZRows z;
  z.off[0] = kb - kb / 4 * 4;
  z.off[1] = (ke - P) - (ke - P) / 4 * 4;
  z.pitch = (std::max(z.off[0], z.off[1]) + P + 3) / 4 * 4;
  return z;
}

struct JobPlan {
  size_t total;
  size_t off_f[2][6], off_cb[3], off_kd[6], off_rkd[6], off_be, off_ce, off_bh, off_ch;
  size_t off_psi[2][6][3][2];
  size_t off_jsrc, off_tw[4], off_ring, off_acc, off_state, off_tmaps, off_items;
  size_t off_probe, probe_bytes;  // line probe [4][nt][nx] (probe_bytes = 0: none)
  size_t off_mat, off_mtab;       // material index [nx][ny][nzp] and table [256][4] (3D, optional)
  bool mat;
  size_t off_wave;                // ordered form: E-block counts per plane (after 8 spare bytes)
  size_t off_tile;                // 2D tile form: sub-blocks completed per tile [kTileMaxBlocks]
  size_t off_pow;                 // port power [nf] complex float64
  long long N, plane;
  int K, esz, nzp, nbuf, variant, L, nitems;
  int rows;  // 3D per-cell tile rows
  int psi_pitch;  // row length along z of the 3D x- and y-slab psi arrays (nz or nzp)
  int psz;        // row length of the 3D z-slab psi arrays (P, or the vector form's padded rows) ...
  int zoff[2];    // ... and the place of slab cell d = 0 in a row, per side
};

// Flags of the work item whose E box starts at (y0 - 1, z0 - 1) (rows
// y0-1 .. y0+EYB-2, columns z0-1 .. z0+EZB-2).
int item_flags(const oidt_job_desc *d, int y0, int z0) {
  const int ylo = y0 - 1, yhi = y0 + EYB - 2, zlo = z0 - 1, zhi = z0 + EZB - 2, P = d->num_cpml;
  auto meets = [](int lo, int hi, int a, int b) { return a <= b && lo <= b && a <= hi; };  // [lo,hi] and [a,b] intersect
  int f = 0;
  if (ylo <= d->jb || yhi >= d->je || zlo <= d->kb || zhi >= d->ke) f |= kItemEdge;
  if (meets(ylo, yhi, d->jb, d->jb + P - 1) || meets(ylo, yhi, d->je - P, d->je - 1)) f |= kItemYSlab;
  if (meets(zlo, zhi, d->kb, d->kb + P - 1) || meets(zlo, zhi, d->ke - P, d->ke - 1)) f |= kItemZSlab;
  if (d->src_field >= 0 && meets(ylo, yhi, d->src_lo[1], d->src_hi[1] - 1) &&
      meets(zlo, zhi, d->src_lo[2] - 1, d->src_hi[2] - 1))  // z - 1: the Hy source also enters at k + 1
    f |= kItemSrc;
  for (int q = 0; q < 2; ++q)
    if (meets(z0, zhi, d->port_pos[q], d->port_pos[q] + 1)) f |= kItemPort;
  return f;
}

// Relative cost of a tile's plane: general planes run the range tests and
// the CPML updates of their slabs.
double tile_weight(int flags) {
  double w = 1.0;
  if (flags) w += 0.6;
  if (flags & (kItemYSlab | kItemZSlab)) w += 0.8;
  return w;
}

// Work items of one 3D job: tiles of TY x TZ cells in (y, z), chunks of L
// planes in x over the updated planes [ib, ie).  Tiles are ordered by
// decreasing weight (the block scheduler then fills the last wave with cheap
// tiles), the chunks of one tile are adjacent (their shared halo planes are
// read while still in L2).
std::vector<SweepItem> sweep_items(const oidt_job_desc *d, int L) {
  struct Tile { int y0, z0, f; double w; };
  std::vector<Tile> tiles;
  for (int y0 = 0; y0 < d->ny; y0 += TY)
    for (int z0 = 0; z0 < d->nz; z0 += TZ) {
      const int f = item_flags(d, y0, z0);
      tiles.push_back({y0, z0, f, tile_weight(f)});
    }
  std::stable_sort(tiles.begin(), tiles.end(), [](const Tile &a, const Tile &b) { return a.w > b.w; });
  std::vector<SweepItem> v;
  for (const Tile &t : tiles)
    for (int x0 = d->ib; x0 < d->ie; x0 += L) v.push_back({t.y0, t.z0, x0, std::min(x0 + L, d->ie), t.f, 0, 0, 0});
  return v;
}

// March depth: the chunk length L minimising the estimated makespan of one
// step, (total plane iterations) / (resident CTAs) + (one item's length);
// an item of L planes iterates L + 1 times (the E halo plane x0 - 1).
// `slots` = SMs x resident CTAs per SM.  A descriptor's reserved[3] > 0
// replaces this estimate (the tuner's measured choice).
int choose_chunk(const oidt_job_desc *d, int slots) {
  const int planes = d->ie - d->ib;
  const long long tiles = (long long)((d->ny + TY - 1) / TY) * ((d->nz + TZ - 1) / TZ);
  double best = 1e300;
  int bestL = planes;
  for (int L = 4; L <= planes; ++L) {
    const long long chunks = (planes + L - 1) / L;
    const double cost = (double)tiles * (planes + chunks) / slots + (L + 1);
    if (cost < best - 1e-9) { best = cost; bestL = L; }
  }
  return bestL;
}

int g_sweep_slots = 0;  // SMs x resident sweep CTAs (set at context creation)

// Split of a 3D row between the vector form's roles: four-cell groups over
// k in [kb + P, ke - P) rounded inward to multiples of 4 (vector role), the
// other four-cell groups of the row (edge role).
VecGeom vec_geom_of(int kb, int ke, int P, int jb, int je, int nzp) {
  VecGeom g;
  g.kz0 = (kb + P + 3) / 4 * 4;
  g.kz1 = (ke - P) / 4 * 4;
  if (g.kz1 <= g.kz0) g.kz0 = g.kz1 = nzp;  // no z-clean group: every cell in the edge role
  g.nvc = (g.kz1 - g.kz0) / 4;
  g.nedge = g.kz0 + (nzp - g.kz1);
  const long long rows = je - jb;
  g.nb_vec = (int)((rows * g.nvc + kVecThreads - 1) / kVecThreads);
  return g;
}
int vec_edge_blocks(const VecGeom &g, int jb, int je) {
  return (int)(((long long)(je - jb) * (g.nedge / 4) + kVecThreads - 1) / kVecThreads);
}
long long vec_blocks_per_plane(const oidt_job_desc *d, int nzp) {
  const VecGeom g = vec_geom_of(d->kb, d->ke, d->num_cpml, d->jb, d->je, nzp);
  return (long long)g.nb_vec + vec_edge_blocks(g, d->jb, d->je);
}

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
  const bool mat = d->mat_idx || d->mat_tab || d->nmat;
  if (mat && (!is3 || !d->mat_idx || !d->mat_tab || d->nmat < 1 || d->nmat > 256))
    return bad("material index: 3D only, with mat_idx, mat_tab and 1 <= nmat <= 256");
  if (!mat)
    for (int c : cb_of(d->mode))
      if (!d->cb[c]) return bad("missing cb array");
  for (int a = 0; a < 6; ++a)
    if (!d->kdx[a] && (is3 || (a != 2 && a != 5))) return bad("missing kappa*dx array");
  const int nalong = is3 ? d->nz : d->nx;
  for (int q = 0; q < 2; ++q)
    if (d->port_pos[q] < 0 || d->port_pos[q] + 1 >= nalong) return bad("port plane out of range");
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
  if (is3) {  // the 3D kernels address a plane and each CPML slab layer set with 32-bit offsets
    const long long lim = 0x7fffffffLL, nzp4 = align_up(d->nz, 4);
    if ((long long)d->ny * nzp4 > lim || (long long)P * d->ny * d->nz > lim || (long long)d->nx * P * d->nz > lim ||
        (long long)d->nx * d->ny * P > lim)
      return bad("grid too large: an x-plane or a CPML slab holds 2^31 or more elements");
  }
  if (d->probe[0] != 0) {
    if (d->probe[0] != 1 || !is3) return bad("probe[0] must be 0, or 1 (3D line probe)");
    if (d->probe[1] < 0 || d->probe[1] + 1 >= d->ny || d->probe[2] < 0 || d->probe[2] + 1 >= d->nz)
      return bad("line probe needs 0 <= y < ny - 1 and 0 <= z < nz - 1");
  } else if (d->probe[1] != 0 || d->probe[2] != 0) {
    return bad("probe[1..2] must be 0 without a probe");
  }
  if (is3 && (d->reserved[0] < kVariantCell || d->reserved[0] > kVariantWave))
    return bad("reserved[0]: 3D launch form 0 to 3");
  if (!is3 && d->reserved[0] != kVariantCell && d->reserved[0] != kVariantTile)
    return bad("reserved[0]: 2D launch form 0 (per-cell) or 4 (tiles)");
  if (d->reserved[1] != 0 && d->reserved[1] != 1) return bad("reserved[1]: 0 or 1");
  const int variant = d->reserved[0];
  if (variant == kVariantTile && tile2d_smem(d->precision == OIDT_F32 ? 4 : 8, P, kTileThreads, kTileThreads) > kTileSmemMax)
    return bad("tile form: num_cpml too large for a block's shared memory");
  if (variant == kVariantTile && ((long long)d->nx * d->ny > 0x7fffffffLL || (long long)d->nx * P > 0x7fffffffLL))
    return bad("tile form: the grid holds 2^31 or more cells");
  const int rows = d->reserved[2] == 0 || variant == kVariantTile ? kRowsDefault : d->reserved[2];
  if (rows != 2 && rows != 4 && rows != 8) return bad("reserved[2]: tile rows 0 (default), 2, 4 or 8");
  if (d->reserved[2] != 0 && !(is3 && variant == kVariantCell) && !(variant == kVariantTile && d->reserved[2] == 1))
    return bad("reserved[2]: the 3D per-cell form's tile rows, or 1 (one launch per sub-block) for the 2D tile form");
  if (d->reserved[3] < 0 || (d->reserved[3] != 0 && !(is3 ? variant == kVariantSweep : variant == kVariantTile)))
    return bad("reserved[3] is >= 0: the 3D plane sweep's march depth or the 2D tile form's steps per launch");
  const int esz = d->precision == OIDT_F32 ? 4 : 8;
  const int nzp = is3 ? (int)align_up(d->nz, 4) : 1;
  const long long N = (long long)d->nx * d->ny * nzp;
  const long long plane = is3 ? (long long)d->nx * d->ny : d->ny;
  int K = d->ring_steps > 0 ? d->ring_steps : kDefaultRing;
  if (K > 4096) return bad("ring_steps too large");
  if (variant == kVariantSweep && (K & 1)) ++K;  // graphs of the sweep end on the parity they start
  const int nbuf = variant == kVariantSweep || variant == kVariantTile ? 2 : 1;
  const bool vec_rows = variant == kVariantVec || variant == kVariantWave;  // the vector form's kernels
  const int psi_pitch = vec_rows ? nzp : d->nz;
  const ZRows zr = vec_rows ? z_rows(d->kb, d->ke, P) : ZRows{P, {0, 0}};
  if (variant == kVariantWave) {  // block counts per plane and step stay in 32-bit counters
    const long long nb = vec_blocks_per_plane(d, nzp);
    if ((long long)(d->nt + 1) * nb > 0x7fffffffLL) return bad("ordered form: nt x blocks per plane >= 2^31");
  }
  if (vec_rows) {  // 32-bit row offsets of the pitched slabs; x-planes on grid.y
    const long long lim = 0x7fffffffLL;
    if ((long long)P * d->ny * nzp > lim || (long long)d->nx * P * nzp > lim || (long long)d->nx * d->ny * zr.pitch > lim)
      return bad("grid too large: a pitched CPML slab holds 2^31 or more elements");
    if (d->ie - d->ib > 65535) return bad("vector form: at most 65535 updated x-planes");
  }
  Layout L;
  memset(pl, 0, sizeof(*pl));
  for (int b = 0; b < nbuf; ++b)
    for (int f : fields_of(d->mode)) pl->off_f[b][f] = L.take(N * esz);
  for (int c : cb_of(d->mode)) pl->off_cb[c] = L.take(N * esz);
  const int dims[3] = {d->nx, d->ny, d->nz};
  for (int a = 0; a < 6; ++a) {
    if (!is3 && (a == 2 || a == 5)) continue;
    // padded to whole 4-element groups (the vector form loads z kappa rows by 16 bytes)
    pl->off_kd[a] = L.take(align_up(dims[a % 3], 4) * esz);
    pl->off_rkd[a] = L.take(align_up(dims[a % 3], 4) * esz);
  }
  pl->off_be = L.take(P * esz);
  pl->off_ce = L.take(P * esz);
  pl->off_bh = L.take(P * esz);
  pl->off_ch = L.take(P * esz);
  for (auto fa : psi_pairs(d->mode))
    for (int b = 0; b < psi_bufs(nbuf, variant, fa.first); ++b)
      for (int sd = 0; sd < 2; ++sd)
        pl->off_psi[b][fa.first][fa.second][sd] =
            L.take(psi_elems(d->mode, fa.second, d->nx, d->ny, d->nz, P, psi_pitch, zr.pitch) * esz);
  pl->off_jsrc = L.take((size_t)d->nt * esz);
  for (int t = 0; t < 4; ++t) pl->off_tw[t] = L.take((size_t)d->nf * d->nt * 8);
  pl->off_ring = L.take((size_t)K * 2 * nslot_of(d->mode) * plane * esz);
  pl->off_acc = L.take((size_t)2 * ncomp_of(d->mode) * d->nf * plane * 16);
  pl->off_state = L.take(64);
  pl->off_pow = L.take((size_t)d->nf * 16);
  if (mat) {
    pl->mat = true;
    pl->off_mat = L.take((size_t)N);
    pl->off_mtab = L.take((size_t)256 * 4 * esz);
  }
  if (variant == kVariantWave) pl->off_wave = L.take(8 + (size_t)4 * (d->ie - d->ib));
  if (variant == kVariantTile) pl->off_tile = L.take((size_t)4 * kTileMaxBlocks);
  if (d->probe[0] == 1) {
    pl->probe_bytes = (size_t)4 * d->nt * d->nx * esz;
    pl->off_probe = L.take(pl->probe_bytes);
  }
  if (variant == kVariantSweep) {
    pl->off_tmaps = L.take(15 * 128);
    pl->L = d->reserved[3] > 0 ? std::min(d->reserved[3], d->ie - d->ib)
                               : choose_chunk(d, g_sweep_slots > 0 ? g_sweep_slots : 148 * 3);
    pl->nitems = (int)sweep_items(d, pl->L).size();
    pl->off_items = L.take((size_t)pl->nitems * sizeof(SweepItem));
  }
  pl->total = L.off;
  pl->N = N;
  pl->plane = plane;
  pl->K = K;
  pl->rows = rows;
  pl->psi_pitch = psi_pitch;
  pl->psz = zr.pitch;
  pl->zoff[0] = zr.off[0];
  pl->zoff[1] = zr.off[1];
  pl->esz = esz;
  pl->nzp = nzp;
  pl->nbuf = nbuf;
  pl->variant = variant;
  return OIDT_OK;
}

struct Job {
  uint64_t id = 0;
  oidt_job_desc d{};
  JobPlan pl{};
  unsigned char *mem = nullptr;
  // pv[b]: view with buffer b old (sweep reads b, writes b^1); pc[b]: in place on b
  Params<float> pvf[2]{}, pcf[2]{};
  Params<double> pvd[2]{}, pcd[2]{};
  FoldParams<float> ff{};
  FoldParams<double> fd{};
  int parity = 0;                                 // buffer holding the current state
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // K-step block starting at parity 0 / 1
  long long graph_launches = 0;                   // kernels per graph replay
  cudaEvent_t ready = nullptr;                    // uploads finished
  cudaEvent_t done = nullptr;                     // last enqueued work finished
  long long steps_enqueued = 0;
  bool busy = false;
  long long wait_cycles = kWaitCycles;  // plane sweep: bound on its tile-load waits
  TileArgs tile{};                      // 2D tile form: tile extents, tiles along y, halo
  int tile_blocks = 0;                  // ... blocks (tiles) of a launch
  bool tile_coop = false;               // ... a ring block is one cooperative launch of sub-blocks
  size_t tile_smem = 0;                 // ... shared memory of a block
};

constexpr int kAuxStreams = 64;  // a served request is two jobs; the mix keeps ~40 active

}  // namespace

struct oidt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;  // compute
  cudaStream_t upload = nullptr;  // job creation copies
  cudaStream_t readout = nullptr; // port-power reductions (never queued behind compute)
  cudaStream_t aux[kAuxStreams] = {};  // branches of multi-job blocks
  cudaEvent_t fork = nullptr, join[kAuxStreams] = {};
  uint64_t budget = 0, in_use = 0;
  std::map<uint64_t, Job *> jobs;
  uint64_t next_id = 1;
  std::mutex mu;
  std::string err;
  long long launches = 0;
  int sms = 148;      // streaming multiprocessors of the device
  bool coop = false;  // ... and whether it takes cooperative launches
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

template <typename T> Params<T> *views(Job *j);
template <> Params<float> *views<float>(Job *j) { return j->pvf; }
template <> Params<double> *views<double>(Job *j) { return j->pvd; }
template <typename T> Params<T> *cells(Job *j);
template <> Params<float> *cells<float>(Job *j) { return j->pcf; }
template <> Params<double> *cells<double>(Job *j) { return j->pcd; }
template <typename T> FoldParams<T> &fold_of(Job *j);
template <> FoldParams<float> &fold_of<float>(Job *j) { return j->ff; }
template <> FoldParams<double> &fold_of<double>(Job *j) { return j->fd; }

// ---- tensor maps (TMA descriptors) ----------------------------------------
typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// 3D map over a pitched [nx][ny][nzp] array; box [1][EY+1][EZ+8] (z fastest).
bool encode_map(CUtensorMap *m, void *base, int esz, int nzp, int ny, int nx) {
  EncodeTiled enc = encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nzp, (cuuint64_t)ny, (cuuint64_t)nx};
  const cuuint64_t strides[2] = {(cuuint64_t)nzp * esz, (cuuint64_t)ny * nzp * esz};
  const cuuint32_t box[3] = {(cuuint32_t)SweepGeom<float, EYB, EZB>::BZ, (cuuint32_t)SweepGeom<float, EYB, EZB>::BY, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(m, esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// dt/eps grids of a job created with a material index: cb[c][cell] =
// mtab[mat[cell]][c] for k < nz (the row padding stays zero).
template <typename T> __global__ void k_mat_expand(Params<T> p) {
  const long long n = (long long)p.nx * p.ny * p.nzp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    if (t % p.nzp >= p.nz) continue;
    const T *e = p.mtab + 4 * (int)p.mat[t];
    for (int c = 0; c < 3; ++c) const_cast<T *>(p.cb[c])[t] = e[c];
  }
}

template <typename T> void fill_params(Job *J) {
  const oidt_job_desc &d = J->d;
  const JobPlan &pl = J->pl;
  unsigned char *m = J->mem;
  for (int b = 0; b < 2; ++b) {
    Params<T> &p = cells<T>(J)[b];
    memset(&p, 0, sizeof p);
    p.mode = d.mode;
    p.nx = d.nx; p.ny = d.ny; p.nz = d.nz; p.nzp = pl.nzp;
    p.P = d.num_cpml;
    p.ib = d.ib; p.jb = d.jb; p.kb = d.kb; p.ie = d.ie; p.je = d.je; p.ke = d.ke;
    const int bb = b < pl.nbuf ? b : 0;
    for (int f : fields_of(d.mode)) {
      p.f[f] = reinterpret_cast<T *>(m + pl.off_f[bb][f]);
      p.fn[f] = reinterpret_cast<T *>(m + pl.off_f[pl.nbuf == 2 ? bb ^ 1 : 0][f]);
    }
    for (int c : cb_of(d.mode)) p.cb[c] = reinterpret_cast<const T *>(m + pl.off_cb[c]);
    p.mat = pl.mat ? m + pl.off_mat : nullptr;
    p.mtab = pl.mat ? reinterpret_cast<const T *>(m + pl.off_mtab) : nullptr;
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
    p.rdx = T(1) / p.dx;  // RN(1/dx) in T (EXACT divisions by dx rely on it)
    p.psx = p.psy = pl.psi_pitch;
    p.psz = d.mode == OIDT_MODE_YEE3D ? pl.psz : d.num_cpml;
    p.wait_cycles = J->wait_cycles;
    for (auto fa : psi_pairs(d.mode))
      for (int sd = 0; sd < 2; ++sd) {
        const bool two = psi_bufs(pl.nbuf, pl.variant, fa.first) == 2;
        p.psi[fa.first][fa.second][sd] = reinterpret_cast<T *>(m + pl.off_psi[two ? bb : 0][fa.first][fa.second][sd]) +
                                         (fa.second == AZ ? pl.zoff[sd] : 0);
        p.psin[fa.first][fa.second][sd] = p.psi[fa.first][fa.second][sd];  // in place
      }
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
    // sweep view: read buffer b, write the other; E psi likewise
    Params<T> &v = views<T>(J)[b];
    v = p;
    if (pl.nbuf == 2) {
      for (auto fa : psi_pairs(d.mode))
        if (psi_bufs(pl.nbuf, pl.variant, fa.first) == 2)
          for (int sd = 0; sd < 2; ++sd)
            v.psin[fa.first][fa.second][sd] = reinterpret_cast<T *>(m + pl.off_psi[bb ^ 1][fa.first][fa.second][sd]);
      v.tmap_f = m + pl.off_tmaps + (size_t)bb * 6 * 128;
      v.tmap_cb = m + pl.off_tmaps + 12 * 128;
    }
  }
  FoldParams<T> &fp = fold_of<T>(J);
  memset(&fp, 0, sizeof fp);
  fp.mode = d.mode; fp.nx = d.nx; fp.ny = d.ny; fp.nf = d.nf; fp.nt = d.nt;
  fp.nslot = nslot_of(d.mode); fp.ncomp = ncomp_of(d.mode); fp.plane = pl.plane;
  fp.ring = reinterpret_cast<T *>(m + pl.off_ring);
  fp.acc = reinterpret_cast<double2 *>(m + pl.off_acc);
  for (int t = 0; t < 4; ++t) fp.tw[t] = reinterpret_cast<const double *>(m + pl.off_tw[t]);
  fp.wlo0 = d.win_lo[0]; fp.whi0 = d.win_hi[0]; fp.wlo1 = d.win_lo[1]; fp.whi1 = d.win_hi[1];
  fp.state = reinterpret_cast<int *>(m + pl.off_state);
}

// Host array (dense reference layout) <-> pitched device grid.
int copy_grid_h2d(oidt_ctx *ctx, Job *J, void *dst, const void *src, cudaStream_t st) {
  const JobPlan &pl = J->pl;
  const size_t row = (size_t)J->d.nz * pl.esz, pitch = (size_t)pl.nzp * pl.esz, rows = (size_t)J->d.nx * J->d.ny;
  if (row == pitch)
    CU(ctx, cudaMemcpyAsync(dst, src, row * rows, cudaMemcpyHostToDevice, st));
  else
    CU(ctx, cudaMemcpy2DAsync(dst, pitch, src, row, row, rows, cudaMemcpyHostToDevice, st));
  return OIDT_OK;
}
int copy_grid_d2h(oidt_ctx *ctx, Job *J, void *dst, const void *src) {
  const JobPlan &pl = J->pl;
  const size_t row = (size_t)J->d.nz * pl.esz, pitch = (size_t)pl.nzp * pl.esz, rows = (size_t)J->d.nx * J->d.ny;
  if (row == pitch)
    CU(ctx, cudaMemcpy(dst, src, row * rows, cudaMemcpyDeviceToHost));
  else
    CU(ctx, cudaMemcpy2D(dst, row, src, pitch, row, rows, cudaMemcpyDeviceToHost));
  return OIDT_OK;
}

template <typename T> int upload(oidt_ctx *ctx, Job *J, const oidt_job_desc *src) {
  const oidt_job_desc &d = *src;
  const JobPlan &pl = J->pl;
  unsigned char *m = J->mem;
  cudaStream_t st = ctx->upload;
  CU(ctx, cudaMemsetAsync(m, 0, pl.total, st));
  std::vector<T> tab;
  if (pl.mat) {  // the index (pitched like the grids) and its table; the grids are expanded below
    const size_t row = d.nz, rows = (size_t)d.nx * d.ny;
    const uint8_t *idx = d.mat_idx;
    uint8_t hi = 0;
    for (size_t q = 0; q < row * rows; ++q) hi = std::max(hi, idx[q]);
    if (hi >= d.nmat) return fail(ctx, OIDT_ERR_INVALID, "material index %d >= nmat %d", (int)hi, d.nmat);
    CU(ctx, cudaMemcpy2DAsync(m + pl.off_mat, pl.nzp, idx, row, row, rows, cudaMemcpyHostToDevice, st));
    tab.assign((size_t)256 * 4, T(0));
    const T *src = static_cast<const T *>(d.mat_tab);
    for (int q = 0; q < d.nmat; ++q)
      for (int c = 0; c < 3; ++c) tab[(size_t)q * 4 + c] = src[(size_t)q * 3 + c];
    CU(ctx, cudaMemcpyAsync(m + pl.off_mtab, tab.data(), tab.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  } else {
    for (int c : cb_of(d.mode)) {
      int rc = copy_grid_h2d(ctx, J, m + pl.off_cb[c], d.cb[c], st);
      if (rc) return rc;
    }
  }
  const int dims[3] = {d.nx, d.ny, d.nz};
  std::vector<T> rk;
  for (int a = 0; a < 6; ++a) {
    if (d.mode != OIDT_MODE_YEE3D && (a == 2 || a == 5)) continue;
    const int n = dims[a % 3];
    const T *kd = static_cast<const T *>(d.kdx[a]);
    CU(ctx, cudaMemcpyAsync(m + pl.off_kd[a], kd, n * sizeof(T), cudaMemcpyHostToDevice, st));
    rk.resize(n);
    for (int i = 0; i < n; ++i) rk[i] = (T)1 / kd[i];  // RN(1/kd) in T (EXACT divisions rely on it)
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
  if (pl.mat) {  // dt/eps grids from the index, for the forms and cells that read them
    const Params<T> &p = cells<T>(J)[0];
    const long long n = (long long)d.nx * d.ny * pl.nzp;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_mat_expand<T><<<blocks, 256, 0, st>>>(p);
    CU(ctx, cudaGetLastError());
    ctx->launches += 1;
    CU(ctx, cudaStreamSynchronize(st));  // tab is a host temporary
  }
  if (pl.variant == kVariantSweep) {
    std::vector<CUtensorMap> maps(15);
    for (int b = 0; b < 2; ++b)
      for (int f = 0; f < 6; ++f)
        if (!encode_map(&maps[b * 6 + f], m + pl.off_f[b][f], pl.esz, pl.nzp, d.ny, d.nx))
          return fail(ctx, OIDT_ERR_CUDA, "cuTensorMapEncodeTiled failed (field map)");
    for (int c = 0; c < 3; ++c)
      if (!encode_map(&maps[12 + c], m + pl.off_cb[c], pl.esz, pl.nzp, d.ny, d.nx))
        return fail(ctx, OIDT_ERR_CUDA, "cuTensorMapEncodeTiled failed (cb map)");
    CU(ctx, cudaMemcpyAsync(m + pl.off_tmaps, maps.data(), 15 * sizeof(CUtensorMap), cudaMemcpyHostToDevice, st));
    std::vector<SweepItem> it = sweep_items(&d, pl.L);
    CU(ctx, cudaMemcpyAsync(m + pl.off_items, it.data(), it.size() * sizeof(SweepItem), cudaMemcpyHostToDevice, st));
    CU(ctx, cudaStreamSynchronize(st));  // maps and items are host temporaries
  }
  CU(ctx, cudaEventRecord(J->ready, st));
  // Host buffers are borrowed only for this call.
  CU(ctx, cudaStreamSynchronize(st));
  return OIDT_OK;
}

// Launch of a time-step kernel with programmatic stream serialization: the
// kernel may be scheduled while its predecessor in the stream drains, and
// waits for it in pdl_wait() (every step kernel calls it first).  This hides
// the gap between dependent launches, which dominates small grids.
template <typename... KArgs, typename... Args>
void launch_step_kernel(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                        Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// One 3D per-cell half-step (H = false: E, true: H) with blocks of 32 x BY
// cells; pdl = false launches without the programmatic-serialization
// attribute (the per-launch timing path).
template <typename T, bool EXACT, int BY>
void y3_half_by(bool H, bool pdl, const Params<T> &p, int s, cudaStream_t st) {
  const dim3 blk(kBlock3Z, BY), grd((p.nz + kBlock3Z - 1) / kBlock3Z, (p.ny + BY - 1) / BY, p.nx);
  void (*kern)(Params<T>, int) = H ? k_y3_h<T, EXACT, BY> : k_y3_e<T, EXACT, BY>;
  if (pdl) launch_step_kernel(kern, grd, blk, 0, st, p, s);
  else kern<<<grd, blk, 0, st>>>(p, s);
}
template <typename T, bool EXACT>
void y3_half(int rows, bool H, bool pdl, const Params<T> &p, int s, cudaStream_t st) {
  if (rows == 2) y3_half_by<T, EXACT, 2>(H, pdl, p, s, st);
  else if (rows == 8) y3_half_by<T, EXACT, 8>(H, pdl, p, s, st);
  else y3_half_by<T, EXACT, 4>(H, pdl, p, s, st);
}

template <typename T> VecGeom vec_geom(const Params<T> &p) { return vec_geom_of(p.kb, p.ke, p.P, p.jb, p.je, p.nzp); }

// One 3D vector-form half-step: the vector-role blocks, then the edge-role
// blocks, of one x-plane per grid row.
template <typename T, bool EXACT> void v3_half(bool H, bool pdl, const Params<T> &p, int s, cudaStream_t st) {
  const VecGeom g = vec_geom(p);
  const long long nb_edge = vec_edge_blocks(g, p.jb, p.je);
  const dim3 grd((unsigned)(g.nb_vec + nb_edge), p.ie - p.ib), blk(kVecThreads);
  void (*kern)(Params<T>, VecGeom, int) = H ? k_v3_h<T, EXACT> : k_v3_e<T, EXACT>;
  if (pdl) launch_step_kernel(kern, grd, blk, 0, st, p, g, s);
  else kern<<<grd, blk, 0, st>>>(p, g, s);
}

// One time step of the ordered form: both half-steps, plane by plane, in one
// launch of 2 (ie - ib) blocks per plane and half-step (k_v3_wave).
// The ordered form's lag: as many planes as keep the arrays a plane of the
// step touches (six fields, the dt/eps grids) within 32 MB of L2, 2 to 32.
template <typename T> int wave_lag(const Params<T> &p) {
  const double plane = (double)p.ny * p.nzp * sizeof(T) * 9;
  const int n = p.ie - p.ib;
  return std::max(1, std::min(n, std::max(2, std::min(32, (int)(32.0e6 / plane)))));
}

template <typename T, bool EXACT> void v3_wave(Job *J, bool pdl, const Params<T> &p, int s, cudaStream_t st) {
  const VecGeom g = vec_geom(p);
  WaveArgs w;
  w.done = reinterpret_cast<int *>(J->mem + J->pl.off_wave + 8);
  w.nb = g.nb_vec + vec_edge_blocks(g, p.jb, p.je);
  w.lag = wave_lag(p);
  const dim3 grd((unsigned)(2LL * (p.ie - p.ib) * w.nb)), blk(kVecThreads);
  if (pdl) launch_step_kernel(k_v3_wave<T, EXACT>, grd, blk, 0, st, p, g, w, s);
  else k_v3_wave<T, EXACT><<<grd, blk, 0, st>>>(p, g, w, s);
}

// One launch of the 2D tile form (k_2d_tile): steps s0 .. s0 + cnt - 1 of a
// ring block, read from buffer p.f / p.psi, owned cells written to p.fn /
// p.psin.
// cnt > halo: one cooperative launch of ceil(cnt / halo) sub-blocks.
template <typename T, bool EXACT>
void tile_launch(bool pdl, Job *J, const Params<T> &p, int s0, int cnt, cudaStream_t st) {
  void (*kern)(Params<T>, TileArgs) =
      p.mode == OIDT_MODE_TM2 ? k_2d_tile<T, EXACT, OIDT_MODE_TM2> : k_2d_tile<T, EXACT, OIDT_MODE_TE2>;
  TileArgs a = J->tile;
  a.s0 = s0;
  a.cnt = cnt;
  a.epoch = reinterpret_cast<int *>(J->mem + J->pl.off_tile);
  if (cnt > a.halo) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(J->tile_blocks);
    cfg.blockDim = dim3(kTileThreads);
    cfg.dynamicSmemBytes = J->tile_smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, p, a);
  } else if (pdl) {
    launch_step_kernel(kern, dim3(J->tile_blocks), dim3(kTileThreads), J->tile_smem, st, p, a);
  } else {
    kern<<<J->tile_blocks, kTileThreads, J->tile_smem, st>>>(p, a);
  }
}

// Launches of the 2D tile form for cnt steps: up to halo steps each.
int tile_launches(const Job *J, int cnt) { return (cnt + J->tile.halo - 1) / J->tile.halo; }

template <typename T> size_t sweep_smem() { return sweep_smem_bytes<T, EYB, EZB, ST>(); }

template <typename T, bool EXACT>
void launch_sweep(const Params<T> &p, const SweepItem *items, int nitems, int s, cudaStream_t st) {
  launch_step_kernel(k_sweep3d<T, EXACT, EYB, EZB, ST>, dim3(nitems), dim3(SweepGeom<T, EYB, EZB>::THREADS),
                     sweep_smem<T>(), st, p, items, s);
}

// One time step of one job (s = step offset inside the K block, par = the
// buffer holding the state at this step).
// Line probe of the state after step s; `b` = the buffer holding it.
template <typename T, bool EXACT> void launch_probe(oidt_ctx *ctx, Job *J, int s, int b, cudaStream_t st) {
  const Params<T> &p = cells<T>(J)[b];
  ProbeArgs<T> a;
  a.ey = p.f[EY];
  a.ez = p.f[EZ];
  a.hy = p.f[HY];
  a.hz = p.f[HZ];
  a.out = reinterpret_cast<T *>(J->mem + J->pl.off_probe);
  a.nx = J->d.nx;
  a.nt = J->d.nt;
  a.ie = J->d.ie;
  a.jc = J->d.probe[1];
  a.kc = J->d.probe[2];
  a.sy = J->pl.nzp;
  a.sx = (long long)J->d.ny * J->pl.nzp;
  a.state = reinterpret_cast<const int *>(J->mem + J->pl.off_state);
  launch_step_kernel(k_probe<T, EXACT>, dim3((a.ie + 127) / 128), dim3(128), 0, st, a, s);
  ctx->launches += 1;
}

template <typename T, bool EXACT> void launch_step(oidt_ctx *ctx, Job *J, int s, int par, cudaStream_t st) {
  if (J->pl.variant == kVariantSweep) {
    launch_sweep<T, EXACT>(views<T>(J)[par], reinterpret_cast<const SweepItem *>(J->mem + J->pl.off_items),
                           J->pl.nitems, s, st);
    ctx->launches += 1;
    if (J->pl.probe_bytes) launch_probe<T, EXACT>(ctx, J, s, par ^ 1, st);
    return;
  }
  Params<T> &p = cells<T>(J)[par];
  if (J->pl.variant == kVariantWave) {
    v3_wave<T, EXACT>(J, true, p, s, st);
    ctx->launches += 1;
    if (J->pl.probe_bytes) launch_probe<T, EXACT>(ctx, J, s, par, st);
    return;
  }
  if (J->pl.variant == kVariantVec) {
    v3_half<T, EXACT>(false, true, p, s, st);
    v3_half<T, EXACT>(true, true, p, s, st);
  } else if (J->d.mode == OIDT_MODE_YEE3D) {
    y3_half<T, EXACT>(J->pl.rows, false, true, p, s, st);
    y3_half<T, EXACT>(J->pl.rows, true, true, p, s, st);
  } else {
    dim3 blk(kBlock2), grd((p.ny + kBlock2 - 1) / kBlock2, p.nx);
    launch_step_kernel(k_2d_e<T, EXACT>, grd, blk, 0, st, p, s);
    launch_step_kernel(k_2d_h<T, EXACT>, grd, blk, 0, st, p, s);
  }
  ctx->launches += 2;
  if (J->pl.probe_bytes) launch_probe<T, EXACT>(ctx, J, s, par, st);
}

template <typename T, bool EXACT> void launch_fold(oidt_ctx *ctx, Job *J, int count, cudaStream_t st) {
  FoldParams<T> &fp = fold_of<T>(J);
  const int wj = fp.whi1 - fp.wlo1;
  const int wi = J->d.mode == OIDT_MODE_YEE3D ? fp.whi0 - fp.wlo0 : 1;
  if (J->d.mode == OIDT_MODE_YEE3D) {
    dim3 grd((wi * wj + 127) / 128, (fp.nf + kFoldF - 1) / kFoldF, 2 * fp.ncomp);
    launch_step_kernel(k_fold<T, EXACT, kFoldF>, grd, dim3(128), 0, st, fp, count);
  } else {
    dim3 grd((wi * wj + 127) / 128, fp.nf, 2 * fp.ncomp);
    launch_step_kernel(k_fold<T, EXACT, 1>, grd, dim3(128), 0, st, fp, count);
  }
  ctx->launches += 1;
}

int steps_flip(const Job *J) { return J->pl.variant == kVariantSweep ? 1 : 0; }

// Buffer parity change of a cnt-step block: the plane sweep flips every step,
// the tile form every launch.
int block_flip(const Job *J, int cnt) {
  if (J->pl.variant == kVariantSweep) return cnt & 1;
  if (J->pl.variant == kVariantTile) return tile_launches(J, cnt) & 1;
  return 0;
}

// Steps 0..cnt-1 of a K-step block starting on buffer parity par.
template <typename T, bool EXACT> void launch_steps(oidt_ctx *ctx, Job *J, int cnt, int par, cudaStream_t st) {
  if (J->pl.variant == kVariantTile) {  // each sub-block reads one buffer and writes the other
    if (J->tile_coop) {
      tile_launch<T, EXACT>(true, J, views<T>(J)[par], 0, cnt, st);
      ctx->launches += 1;
      return;
    }
    const int nl = tile_launches(J, cnt);
    for (int l = 0; l < nl; ++l) {
      const int s0 = l * J->tile.halo;
      tile_launch<T, EXACT>(true, J, views<T>(J)[par ^ (l & 1)], s0, std::min(J->tile.halo, cnt - s0), st);
    }
    ctx->launches += nl;
    return;
  }
  const int flip = steps_flip(J);
  for (int s = 0; s < cnt; ++s) launch_step<T, EXACT>(ctx, J, s, par ^ (flip & s), st);
}

// The job's K-step block starting on buffer parity par (its steps, then its
// DFT fold) as a CUDA graph, captured on stream st at first use.  Capture
// enqueues nothing, so st may hold work of other jobs.
template <typename T, bool EXACT> int job_graph(oidt_ctx *ctx, Job *J, int par, cudaStream_t st) {
  if (J->graph[par]) return OIDT_OK;
  const int K = J->pl.K;
  cudaGraph_t g;
  const long long before = ctx->launches;
  CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  launch_steps<T, EXACT>(ctx, J, K, par, st);
  launch_fold<T, EXACT>(ctx, J, K, st);
  CU(ctx, cudaStreamEndCapture(st, &g));
  const cudaError_t ie = cudaGraphInstantiate(&J->graph[par], g, 0);
  cudaGraphDestroy(g);
  CU(ctx, ie);
  J->graph_launches = ctx->launches - before;
  ctx->launches = before;
  return OIDT_OK;
}

template <typename T, bool EXACT> int advance_t(oidt_ctx *ctx, Job *J, int nsteps) {
  cudaStream_t st = ctx->stream;
  CU(ctx, cudaStreamWaitEvent(st, J->ready, 0));
  const int K = J->pl.K;
  int left = nsteps;
  while (left > 0) {
    const int cnt = std::min(K, left);
    const int par = J->parity;
    if (cnt == K && J->d.reserved[1] == 0) {
      int rc = job_graph<T, EXACT>(ctx, J, par, st);
      if (rc) return rc;
      CU(ctx, cudaGraphLaunch(J->graph[par], st));
      ctx->launches += J->graph_launches;
    } else {
      launch_steps<T, EXACT>(ctx, J, cnt, par, st);
      launch_fold<T, EXACT>(ctx, J, cnt, st);
    }
    J->parity ^= block_flip(J, cnt);
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
// A block of cnt steps for several jobs: each job's launches go to one of the
// auxiliary streams, forked from and joined back into the compute stream, so
// independent jobs run concurrently.  A full K-step block of a job is its own
// CUDA graph (the graph single-job advances replay), so a group whose
// membership changes from one call to the next -- a serving loop's groups do
// at every admission and retirement -- costs no capture; launches of one
// graph are ordered by CUDA even when they go to different streams.
template <typename T, bool EXACT> int batch_block(oidt_ctx *ctx, std::vector<Job *> &js, int cnt, cudaStream_t st) {
  const bool full = cnt == js[0]->pl.K;
  if (full)  // capture missing graphs before the fork (capture enqueues nothing)
    for (Job *J : js)
      if (J->d.reserved[1] == 0) {
        int rc = job_graph<T, EXACT>(ctx, J, J->parity, st);
        if (rc) return rc;
      }
  const int na = std::min<int>(kAuxStreams, (int)js.size());
  CU(ctx, cudaEventRecord(ctx->fork, st));
  for (int a = 0; a < na; ++a) CU(ctx, cudaStreamWaitEvent(ctx->aux[a], ctx->fork, 0));
  for (int b = 0; b < (int)js.size(); ++b) {
    Job *J = js[b];
    cudaStream_t sb = ctx->aux[b % na];
    if (full && J->d.reserved[1] == 0) {
      CU(ctx, cudaGraphLaunch(J->graph[J->parity], sb));
      ctx->launches += J->graph_launches;
    } else {
      launch_steps<T, EXACT>(ctx, J, cnt, J->parity, sb);
      launch_fold<T, EXACT>(ctx, J, cnt, sb);
    }
    J->parity ^= block_flip(J, cnt);
  }
  for (int a = 0; a < na; ++a) {
    CU(ctx, cudaEventRecord(ctx->join[a], ctx->aux[a]));
    CU(ctx, cudaStreamWaitEvent(st, ctx->join[a], 0));
  }
  return OIDT_OK;
}

template <typename T, bool EXACT>
int batch_t(oidt_ctx *ctx, std::vector<Job *> &js, int nsteps) {
  cudaStream_t st = ctx->stream;
  const int K = js[0]->pl.K;
  for (Job *j : js) {
    if (j->pl.K != K) return fail(ctx, OIDT_ERR_INVALID, "batched jobs must share ring_steps");
    CU(ctx, cudaStreamWaitEvent(st, j->ready, 0));
  }
  for (int left = nsteps; left > 0;) {
    const int cnt = std::min(K, left);
    int rc = batch_block<T, EXACT>(ctx, js, cnt, st);
    if (rc) return rc;
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

template <typename T, bool EXACT> int profile_t(oidt_ctx *ctx, Job *J, int nsteps, float *ms) {
  cudaStream_t st = ctx->stream;
  CU(ctx, cudaStreamWaitEvent(st, J->ready, 0));
  std::vector<cudaEvent_t> ev(2 * (2 * nsteps + 2));
  for (auto &e : ev) CU(ctx, cudaEventCreate(&e));
  if (J->pl.variant == kVariantTile) {  // launches of up to halo steps: time per step as the E half, H half = 0
    const int nl = tile_launches(J, nsteps);
    cudaEventRecord(ev[0], st);
    if (J->tile_coop) {
      tile_launch<T, EXACT>(false, J, views<T>(J)[J->parity], 0, nsteps, st);
    } else {
      for (int l = 0; l < nl; ++l) {
        const int s0 = l * J->tile.halo;
        tile_launch<T, EXACT>(false, J, views<T>(J)[J->parity ^ (l & 1)], s0, std::min(J->tile.halo, nsteps - s0), st);
      }
    }
    cudaEventRecord(ev[1], st);
    launch_fold<T, EXACT>(ctx, J, nsteps, st);
    cudaEventRecord(ev[2], st);
    ctx->launches += J->tile_coop ? 1 : nl;
    J->parity ^= nl & 1;
    CU(ctx, cudaGetLastError());
    CU(ctx, cudaStreamSynchronize(st));
    float a = 0, fo = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&fo, ev[1], ev[2]);
    ms[0] = a / nsteps;
    ms[1] = 0;
    ms[2] = fo;
    for (auto &e : ev) cudaEventDestroy(e);
    J->steps_enqueued += nsteps;
    CU(ctx, cudaEventRecord(J->done, st));
    return OIDT_OK;
  }
  const bool sweep = J->pl.variant == kVariantSweep;
  int q = 0;
  for (int s = 0; s < nsteps; ++s) {
    const int par = J->parity ^ (sweep ? (s & 1) : 0);
    if (sweep) {  // one launch per step: reported as the E half, H half = 0
      cudaEventRecord(ev[q++], st);
      launch_sweep<T, EXACT>(views<T>(J)[par], reinterpret_cast<const SweepItem *>(J->mem + J->pl.off_items),
                             J->pl.nitems, s, st);
      ctx->launches += 1;
      cudaEventRecord(ev[q++], st);
      cudaEventRecord(ev[q++], st);
      cudaEventRecord(ev[q++], st);
      if (J->pl.probe_bytes) launch_probe<T, EXACT>(ctx, J, s, par ^ 1, st);  // untimed
      continue;
    }
    Params<T> &p = cells<T>(J)[par];
    if (J->pl.variant == kVariantWave) {  // one launch per step: reported as the E half, H half = 0
      cudaEventRecord(ev[q++], st);
      v3_wave<T, EXACT>(J, false, p, s, st);
      cudaEventRecord(ev[q++], st);
      cudaEventRecord(ev[q++], st);
      cudaEventRecord(ev[q++], st);
      ctx->launches += 1;
      if (J->pl.probe_bytes) launch_probe<T, EXACT>(ctx, J, s, par, st);  // untimed
      continue;
    }
    if (J->d.mode == OIDT_MODE_YEE3D) {
      const bool vec = J->pl.variant == kVariantVec;
      cudaEventRecord(ev[q++], st);
      if (vec) v3_half<T, EXACT>(false, false, p, s, st);
      else y3_half<T, EXACT>(J->pl.rows, false, false, p, s, st);
      cudaEventRecord(ev[q++], st);
      cudaEventRecord(ev[q++], st);
      if (vec) v3_half<T, EXACT>(true, false, p, s, st);
      else y3_half<T, EXACT>(J->pl.rows, true, false, p, s, st);
      cudaEventRecord(ev[q++], st);
      if (J->pl.probe_bytes) launch_probe<T, EXACT>(ctx, J, s, par, st);  // untimed
    } else {
      dim3 blk(kBlock2), grd((p.ny + kBlock2 - 1) / kBlock2, p.nx);
      cudaEventRecord(ev[q++], st);
      k_2d_e<T, EXACT><<<grd, blk, 0, st>>>(p, s);
      cudaEventRecord(ev[q++], st);
      cudaEventRecord(ev[q++], st);
      k_2d_h<T, EXACT><<<grd, blk, 0, st>>>(p, s);
      cudaEventRecord(ev[q++], st);
    }
    ctx->launches += 2;
  }
  cudaEventRecord(ev[q++], st);
  launch_fold<T, EXACT>(ctx, J, nsteps, st);
  cudaEventRecord(ev[q++], st);
  CU(ctx, cudaGetLastError());
  CU(ctx, cudaStreamSynchronize(st));
  double se = 0, sh = 0;
  for (int s = 0; s < nsteps; ++s) {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ev[4 * s], ev[4 * s + 1]);
    cudaEventElapsedTime(&b, ev[4 * s + 2], ev[4 * s + 3]);
    se += a;
    sh += b;
  }
  float fo = 0;
  cudaEventElapsedTime(&fo, ev[4 * nsteps], ev[4 * nsteps + 1]);
  ms[0] = (float)(se / nsteps);
  ms[1] = (float)(sh / nsteps);
  ms[2] = fo;
  for (auto &e : ev) cudaEventDestroy(e);
  if (sweep) J->parity ^= nsteps & 1;
  J->steps_enqueued += nsteps;
  CU(ctx, cudaEventRecord(J->done, st));
  return OIDT_OK;
}

void destroy_job(oidt_ctx *ctx, Job *J) {
  for (int b = 0; b < 2; ++b)
    if (J->graph[b]) cudaGraphExecDestroy(J->graph[b]);
  cudaFreeAsync(J->mem, ctx->stream);  // stream-ordered: no device-wide synchronisation
  cudaEventDestroy(J->ready);
  cudaEventDestroy(J->done);
  delete J;
}

int set_sweep_attrs() {
  cudaFuncSetAttribute(k_sweep3d<float, false, EYB, EZB, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem<float>());
  // (each launch passes its job's parameters by value: about 1 KB of kernel parameter space)
  cudaFuncSetAttribute(k_sweep3d<float, true, EYB, EZB, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem<float>());
  cudaFuncSetAttribute(k_sweep3d<double, false, EYB, EZB, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem<double>());
  cudaFuncSetAttribute(k_sweep3d<double, true, EYB, EZB, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem<double>());
  int per_sm = 0, sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep3d<float, false, EYB, EZB, ST>, SweepGeom<float, EYB, EZB>::THREADS, sweep_smem<float>());
  return std::max(1, per_sm) * std::max(1, sms);
}

// The 2D tile kernels take tile2d_smem(esz, P) bytes of shared memory a block, at
// most kTileSmemMax.
template <typename T, bool EXACT, int MODE> void tile_attrs_of() {
  cudaFuncSetAttribute(k_2d_tile<T, EXACT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmemMax);
}

void set_tile_attrs() {
  tile_attrs_of<float, false, OIDT_MODE_TM2>();
  tile_attrs_of<float, true, OIDT_MODE_TM2>();
  tile_attrs_of<double, false, OIDT_MODE_TM2>();
  tile_attrs_of<double, true, OIDT_MODE_TM2>();
  tile_attrs_of<float, false, OIDT_MODE_TE2>();
  tile_attrs_of<float, true, OIDT_MODE_TE2>();
  tile_attrs_of<double, false, OIDT_MODE_TE2>();
  tile_attrs_of<double, true, OIDT_MODE_TE2>();
}

// The tile form's split of a job.  A held tile has at most kTileThreads
// cells.  For each steps-per-launch h (the halo: at most min(8, ring steps),
// or the descriptor's reserved[3]), the tiling with the fewest waves of blocks
// over the SMs, then the fewest cells held in all; then the h with the least
// estimated time per step: about 0.5 us per step and wave, and about 2 us of
// launch overhead per launch.
void tile_plan(Job *J, int sms) {
  const oidt_job_desc &d = J->d;
  const int nx = d.nx, ny = d.ny;
  const int hmax = std::min(kTileHaloMax, J->pl.K);
  const int h0 = d.reserved[3] > 0 ? std::min(d.reserved[3], hmax) : 1;
  const int h1 = d.reserved[3] > 0 ? h0 : hmax;
  double best_t = 1e30;
  for (int h = h0; h <= h1; ++h) {
    long long bk0 = -1, bk1 = 0;
    TileArgs bt{};
    int bb = 0;
    // a held tile of (ti + 2h) x (tj + 2h) <= kTileThreads cells (clipped at the grid's edges)
    for (int ti = 1; ti <= nx; ++ti) {
      const int hi = std::min(nx, ti + 2 * h);
      if (hi > kTileThreads) break;
      const int gi = (nx + ti - 1) / ti;
      if (ti > 1 && (nx + ti - 2) / (ti - 1) == gi) continue;  // the smallest ti of this tile count
      // the widest owned tile, then the narrowest with as many tiles along y
      const int tjmax = ny * hi <= kTileThreads ? ny : std::min(ny, kTileThreads / hi - 2 * h);
      if (tjmax < 1) continue;
      const int gjn = (ny + tjmax - 1) / tjmax;
      {
        const int tj = (ny + gjn - 1) / gjn;
        const long long tiles = (long long)gi * ((ny + tj - 1) / tj);
        const long long cells = (long long)std::min(nx, ti + 2 * h) * std::min(ny, tj + 2 * h);
        const long long k0 = (tiles + sms - 1) / sms, k1 = tiles * cells;
        if (bk0 < 0 || k0 < bk0 || (k0 == bk0 && k1 < bk1)) {
          bk0 = k0;
          bk1 = k1;
          bt.ti = ti;
          bt.tj = tj;
          bt.gj = (ny + tj - 1) / tj;
          bb = (int)tiles;
        }
      }
    }
    if (bk0 < 0) continue;
    const double t = 0.5 * (double)bk0 + 2.0 / h;
    if (t < best_t) {
      best_t = t;
      J->tile = bt;
      J->tile.halo = h;
      J->tile_blocks = bb;
    }
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
// ---- capture ring refill after a field write ----------------------------------
// The update kernels write a component's sample into the capture ring only
// where they update it; cells a step never updates (the PEC rim) keep their
// value for the whole run, and the fold's colocation reaches them when the DFT
// window touches the rim (a one-cell CPML).  After fields are written, every
// ring slot is filled with the current port-plane values, so the slots no
// update overwrites hold those constant values.  Slots: 3D Ex, Ey, Hx(k),
// Hx(k+1), Hy(k), Hy(k+1) on the z = port planes; TM2 Ez, Hy(x), Hy(x+1) and
// TE2 Ey, Hz(x), Hz(x+1) on the x = port planes.
namespace {
template <typename T> __global__ void k_ring_fill(Params<T> p) {
  const long long n = (long long)p.ring_K * 2 * p.nslot * p.plane;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long c = t % p.plane, r = t / p.plane;
    const int slot = (int)(r % p.nslot), q = (int)((r / p.nslot) % 2);
    const int port = p.port_pos[q];
    T v;
    if (p.mode == OIDT_MODE_YEE3D) {
      const int f = slot == 0 ? EX : slot == 1 ? EY : slot < 4 ? HX : HY;
      const int d = (slot == 3 || slot == 5) ? 1 : 0;
      v = p.f[f][c * p.nzp + port + d];
    } else {
      const int f = slot == 0 ? (p.mode == OIDT_MODE_TM2 ? EZ : EY) : (p.mode == OIDT_MODE_TM2 ? HY : HZ);
      const int d = slot == 2 ? 1 : 0;
      v = p.f[f][(long long)(port + d) * p.ny + c];
    }
    p.ring[t] = v;
  }
}
}  // namespace

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
      cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->readout, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return OIDT_ERR_CUDA;
  }
  for (int a = 0; a < kAuxStreams; ++a) {
    cudaStreamCreateWithFlags(&ctx->aux[a], cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&ctx->join[a], cudaEventDisableTiming);
  }
  cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming);
  g_sweep_slots = set_sweep_attrs();
  set_tile_attrs();
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  ctx->coop = coop != 0;
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
    for (auto &kv : ctx->jobs) destroy_job(ctx, kv.second);
    ctx->jobs.clear();
    cudaStreamSynchronize(ctx->stream);
    for (int a = 0; a < kAuxStreams; ++a) {
      cudaStreamSynchronize(ctx->aux[a]);
      cudaStreamDestroy(ctx->aux[a]);
      cudaEventDestroy(ctx->join[a]);
    }
    cudaEventDestroy(ctx->fork);
    cudaStreamSynchronize(ctx->readout);
    cudaStreamDestroy(ctx->stream);
    cudaStreamDestroy(ctx->upload);
    cudaStreamDestroy(ctx->readout);
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
  if (pl.variant == kVariantTile) {
    tile_plan(J, ctx->sms);
    J->tile_smem = tile2d_smem(pl.esz, desc->num_cpml, J->tile.ti + 2 * J->tile.halo, J->tile.tj + 2 * J->tile.halo);
    // a ring block in one launch where every tile is resident at once and a tile's
    // halo reaches its 8 neighbours only
    J->tile_coop = ctx->coop && desc->reserved[2] == 0 && J->tile_blocks <= std::min(ctx->sms, kTileMaxBlocks) &&
                   J->tile.halo <= std::min(J->tile.ti, J->tile.tj) && J->pl.K > J->tile.halo;
  }
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
  J->d.mat_idx = nullptr;
  J->d.mat_tab = nullptr;
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
    for (Job *o : js)
      if (o == J) return fail(ctx, OIDT_ERR_INVALID, "job %llu listed twice", (unsigned long long)jobs[b]);
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
  int *state = nullptr;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    Job *J = find(ctx, job);
    if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
    if (!J->busy) return OIDT_OK;
    ev = J->done;
    state = reinterpret_cast<int *>(J->mem + J->pl.off_state);
  }
  cudaSetDevice(ctx->device);
  int rc = wait_event(ctx, ev, timeout_ms);
  if (rc == OIDT_OK) {
    std::lock_guard<std::mutex> g(ctx->mu);
    Job *J = find(ctx, job);
    if (J && J->done == ev) J->busy = cudaEventQuery(ev) != cudaSuccess;
    int flags[2] = {0, 0};
    if (cudaMemcpy(flags, state, sizeof flags, cudaMemcpyDeviceToHost) == cudaSuccess && flags[1])
      return fail(ctx, OIDT_ERR_TIMEOUT,
                  "a kernel's bounded wait expired (device flag %d: 1 = the plane sweep's tile loads, "
                  "2 = the ordered form's plane order, 3 = the 2D tile form's neighbour tiles)", flags[1]);
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

int32_t oidt_job_read_probe(oidt_ctx *ctx, uint64_t job, int32_t comp, void *out, size_t nbytes) {
  if (!ctx || !out) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  if (!J->pl.probe_bytes) return fail(ctx, OIDT_ERR_STATE, "job has no line probe");
  if (comp < 0 || comp > 3) return fail(ctx, OIDT_ERR_INVALID, "probe comp must be 0..3 (Ey, Ez, Hy, Hz)");
  const size_t need = J->pl.probe_bytes / 4;
  if (nbytes < need) return fail(ctx, OIDT_ERR_INVALID, "output needs %zu bytes", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  CU(ctx, cudaMemcpy(out, J->mem + J->pl.off_probe + comp * need, need, cudaMemcpyDeviceToHost));
  return OIDT_OK;
}

// ---- port power: the S-parameter sums, reduced on the device ----------------
// P[f] = sum over the window of the port plane's complex Poynting density in
// float64: 3D 1/2 (Ex Hy* - Ey Hx*) (FDTD_3D extract_sparams.py:114-115), 2D TM
// -1/2 Ez Hy*, 2D TE 1/2 Ey Hz* (FDTD_2D_TM / FDTD_2D_TE extract_sparams.py:
// 88-89), of this job's accumulators or of their difference with another
// job's (the reflected wave).  One block per frequency; each thread sums a
// strided subset of the window, then a fixed-shape tree combines the
// threads, so the result does not depend on scheduling.
namespace {
constexpr int kPowThreads = 256;
struct PowerArgs {
  const double2 *a[4], *b[4];  // b[0] == nullptr: no subtraction
  double2 *out;
  long long plane;
  int cols, i0, j0, wi, wj, mode;
};

__device__ __forceinline__ double2 cmul_conj(double2 u, double2 v) {  // u * conj(v)
  return make_double2(u.x * v.x + u.y * v.y, u.y * v.x - u.x * v.y);
}

__global__ void __launch_bounds__(kPowThreads) k_port_power(PowerArgs a) {
  const int f = blockIdx.x;
  const long long n = (long long)a.wi * a.wj, base = (long long)f * a.plane;
  const int nc = a.mode == OIDT_MODE_YEE3D ? 4 : 2;
  double re = 0.0, im = 0.0;
  for (long long t = threadIdx.x; t < n; t += kPowThreads) {
    const long long o = base + (long long)(a.i0 + (int)(t / a.wj)) * a.cols + (a.j0 + (int)(t % a.wj));
    double2 v[4];
    for (int c = 0; c < nc; ++c) {
      v[c] = a.a[c][o];
      if (a.b[0]) {
        const double2 w = a.b[c][o];
        v[c].x -= w.x;
        v[c].y -= w.y;
      }
    }
    double2 p;
    if (a.mode == OIDT_MODE_YEE3D) {
      const double2 p1 = cmul_conj(v[0], v[3]), p2 = cmul_conj(v[1], v[2]);
      p = make_double2(0.5 * (p1.x - p2.x), 0.5 * (p1.y - p2.y));
    } else {
      const double2 q = cmul_conj(v[0], v[1]);
      const double s = a.mode == OIDT_MODE_TM2 ? -0.5 : 0.5;
      p = make_double2(s * q.x, s * q.y);
    }
    re += p.x;
    im += p.y;
  }
  for (int d = 16; d > 0; d >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, d);
    im += __shfl_down_sync(0xffffffffu, im, d);
  }
  __shared__ double sr[kPowThreads / 32], si[kPowThreads / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sr[w] = re; si[w] = im; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0, i = 0.0;
    for (int q = 0; q < kPowThreads / 32; ++q) { r += sr[q]; i += si[q]; }
    a.out[f] = make_double2(r, i);
  }
}
}  // namespace

int32_t oidt_job_port_power(oidt_ctx *ctx, uint64_t job, uint64_t minus_job, int32_t port, const int32_t *window,
                            double *out, size_t n) {
  if (!ctx || !out || !window) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  Job *M = nullptr;
  if (minus_job) {
    M = find(ctx, minus_job);
    if (!M) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)minus_job);
    if (M == J) return fail(ctx, OIDT_ERR_INVALID, "minus_job is the job itself");
    // the port plane: 3D [nx][ny], 2D [ny] (nx is then the guide length, free)
    if (M->d.mode != J->d.mode || M->d.nf != J->d.nf || M->d.ny != J->d.ny ||
        (J->d.mode == OIDT_MODE_YEE3D && M->d.nx != J->d.nx))
      return fail(ctx, OIDT_ERR_INVALID, "minus_job needs the same mode, nf and port plane");
  }
  if (port < 0 || port > 1) return fail(ctx, OIDT_ERR_INVALID, "bad port");
  const bool is3 = J->d.mode == OIDT_MODE_YEE3D;
  const int rows = is3 ? J->d.nx : 1, cols = J->d.ny;
  const int i0 = window[0], i1 = window[1], j0 = window[2], j1 = window[3];
  if (i0 < 0 || i1 > rows || i0 >= i1 || j0 < 0 || j1 > cols || j0 >= j1)
    return fail(ctx, OIDT_ERR_INVALID, "window must lie in the %d x %d port plane and be non-empty", rows, cols);
  if (n < (size_t)2 * J->d.nf) return fail(ctx, OIDT_ERR_INVALID, "output needs %d doubles", 2 * J->d.nf);
  CU(ctx, cudaSetDevice(ctx->device));
  for (Job *X : {J, M}) {  // uploaded, and every step enqueued so far done
    if (!X) continue;
    CU(ctx, cudaStreamWaitEvent(ctx->readout, X->ready, 0));
    CU(ctx, cudaStreamWaitEvent(ctx->readout, X->done, 0));
  }
  const int nc = ncomp_of(J->d.mode);
  const size_t span = (size_t)J->d.nf * J->pl.plane;
  PowerArgs a = {};
  for (int c = 0; c < nc; ++c) {
    a.a[c] = reinterpret_cast<const double2 *>(J->mem + J->pl.off_acc) + ((size_t)port * nc + c) * span;
    if (M) a.b[c] = reinterpret_cast<const double2 *>(M->mem + M->pl.off_acc) + ((size_t)port * nc + c) * span;
  }
  a.out = reinterpret_cast<double2 *>(J->mem + J->pl.off_pow);
  a.plane = J->pl.plane;
  a.cols = cols;
  a.i0 = i0;
  a.j0 = j0;
  a.wi = i1 - i0;
  a.wj = j1 - j0;
  a.mode = J->d.mode;
  k_port_power<<<J->d.nf, kPowThreads, 0, ctx->readout>>>(a);
  CU(ctx, cudaGetLastError());
  CU(ctx, cudaMemcpyAsync(out, a.out, (size_t)J->d.nf * 16, cudaMemcpyDeviceToHost, ctx->readout));
  CU(ctx, cudaStreamSynchronize(ctx->readout));
  return OIDT_OK;
}

// ---- port-window DFT readout through static device scratch -------------------
// A variant of the staged readout that allocates nothing: the window of one
// (port, component) accumulator is gathered into a file-scope device buffer of
// fixed size and copied to the host from there.  Every element of the
// gathered range is written before it is read, so nothing in the buffer has
// to start at zero.  The buffer is shared by every context on a device, so
// calls on one device must not overlap (calls through one context are
// serialised by its mutex).
namespace {
constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB: 1 Mi complex doubles
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
std::mutex g_static_mu;
constexpr int kMaxDevices = 64;
void *g_static_addr[kMaxDevices] = {};  // resolved once per device

__global__ void k_gather_window(const double2 *__restrict__ acc, double2 *__restrict__ dst, int nf, long long plane,
                                int ny, int i0, int wi, int j0, int wj) {
  const long long n = (long long)nf * wi * wj;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(t % wj);
    const long long r = t / wj;
    const int ii = (int)(r % wi), f = (int)(r / wi);
    dst[t] = acc[f * plane + (long long)(i0 + ii) * ny + (j0 + jj)];
  }
}
}  // namespace

int32_t oidt_job_read_dft_window_static(oidt_ctx *ctx, uint64_t job, int32_t port, int32_t comp, double *out,
                                        size_t n) {
  if (!ctx || !out) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  const int nc = ncomp_of(J->d.mode);
  if (port < 0 || port > 1 || comp < 0 || comp >= nc) return fail(ctx, OIDT_ERR_INVALID, "bad port/comp");
  const bool is3 = J->d.mode == OIDT_MODE_YEE3D;
  const int i0 = is3 ? J->d.win_lo[0] : 0, wi = is3 ? J->d.win_hi[0] - J->d.win_lo[0] : 1;
  const int j0 = J->d.win_lo[1], wj = J->d.win_hi[1] - J->d.win_lo[1];
  const size_t cells = (size_t)J->d.nf * wi * wj, need = 2 * cells;
  if (n < need) return fail(ctx, OIDT_ERR_INVALID, "output needs %zu doubles", need);
  if (need * 8 > kStaticScratchBytes)
    return fail(ctx, OIDT_ERR_INVALID,
                "the DFT window needs %zu bytes of device scratch; the static scratch holds %zu (use oidt_job_read_dft)",
                need * 8, kStaticScratchBytes);
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(ctx, OIDT_ERR_INVALID, "device ordinal out of range");
  int rc = read_common(ctx, J);
  if (rc) return rc;
  void *scratch = nullptr;
  {
    std::lock_guard<std::mutex> gs(g_static_mu);
    if (!g_static_addr[ctx->device]) {
      void *a = nullptr;
      CU(ctx, cudaGetSymbolAddress(&a, g_static_scratch));
      g_static_addr[ctx->device] = a;
    }
    scratch = g_static_addr[ctx->device];
  }
  const double2 *acc = reinterpret_cast<const double2 *>(J->mem + J->pl.off_acc) + ((size_t)port * nc + comp) * J->d.nf * J->pl.plane;
  // on the readout stream: read_common has waited for this job's work, and
  // steps other jobs have queued on the compute stream do not delay the read
  const long long blocks = std::min<long long>((long long)(cells + 255) / 256, 148LL * 8);
  k_gather_window<<<(unsigned)std::max(1LL, blocks), 256, 0, ctx->readout>>>(
      acc, static_cast<double2 *>(scratch), J->d.nf, J->pl.plane, is3 ? J->d.ny : 0, i0, wi, j0, wj);
  CU(ctx, cudaGetLastError());
  ctx->launches += 1;
  CU(ctx, cudaMemcpyAsync(out, scratch, need * 8, cudaMemcpyDeviceToHost, ctx->readout));
  CU(ctx, cudaStreamSynchronize(ctx->readout));
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
  const size_t need = (size_t)J->d.nx * J->d.ny * J->d.nz * J->pl.esz;
  if (nbytes < need) return fail(ctx, OIDT_ERR_INVALID, "output needs %zu bytes", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  return copy_grid_d2h(ctx, J, out, J->mem + J->pl.off_f[J->pl.nbuf == 2 ? J->parity : 0][field]);
}

int32_t oidt_job_write_field(oidt_ctx *ctx, uint64_t job, int32_t field, const void *src, size_t nbytes) {
  if (!ctx || !src) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  if (!field_ok(J, field)) return fail(ctx, OIDT_ERR_INVALID, "field %d not in this solver", field);
  const size_t need = (size_t)J->d.nx * J->d.ny * J->d.nz * J->pl.esz;
  if (nbytes != need) return fail(ctx, OIDT_ERR_INVALID, "input must be %zu bytes", need);
  int rc = read_common(ctx, J);
  if (rc) return rc;
  // Both buffers: cells a step never updates (the PEC rim planes) are not
  // copied between the plane-sweep buffers, so they must agree in both.
  for (int b = 0; b < J->pl.nbuf; ++b) {
    rc = copy_grid_h2d(ctx, J, J->mem + J->pl.off_f[b][field], src, ctx->upload);
    if (rc) return rc;
  }
  const long long n = (long long)J->pl.K * 2 * nslot_of(J->d.mode) * J->pl.plane;
  const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 8);
  if (J->d.precision == OIDT_F64)
    k_ring_fill<double><<<blocks, 256, 0, ctx->upload>>>(cells<double>(J)[J->parity]);
  else
    k_ring_fill<float><<<blocks, 256, 0, ctx->upload>>>(cells<float>(J)[J->parity]);
  CU(ctx, cudaGetLastError());
  ctx->launches += 1;
  CU(ctx, cudaStreamSynchronize(ctx->upload));
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
  const int b = psi_bufs(J->pl.nbuf, J->pl.variant, field) == 2 ? J->parity : 0;
  const unsigned char *src = J->mem + J->pl.off_psi[b][field][axis][side];
  const bool pitched = J->d.mode == OIDT_MODE_YEE3D && axis != AZ && J->pl.psi_pitch != J->d.nz;
  const bool zpitched = J->d.mode == OIDT_MODE_YEE3D && axis == AZ && J->pl.psz != J->d.num_cpml;
  if (pitched) {  // rows of nz cells out of rows of psi_pitch cells
    const size_t row = (size_t)J->d.nz * J->pl.esz, pitch = (size_t)J->pl.psi_pitch * J->pl.esz;
    CU(ctx, cudaMemcpy2D(out, row, src, pitch, row, need / row, cudaMemcpyDeviceToHost));
  } else if (zpitched) {  // rows of P cells out of the padded rows, from the side's first slab cell
    const size_t row = (size_t)J->d.num_cpml * J->pl.esz, pitch = (size_t)J->pl.psz * J->pl.esz;
    CU(ctx, cudaMemcpy2D(out, row, src + (size_t)J->pl.zoff[side] * J->pl.esz, pitch, row, need / row,
                         cudaMemcpyDeviceToHost));
  } else {
    CU(ctx, cudaMemcpy(out, src, need, cudaMemcpyDeviceToHost));
  }
  return OIDT_OK;
}

int32_t oidt_job_release(oidt_ctx *ctx, uint64_t job) {
  if (!ctx) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  CU(ctx, cudaSetDevice(ctx->device));
  CU(ctx, cudaEventSynchronize(J->done));
  ctx->in_use -= J->pl.total;
  ctx->jobs.erase(job);
  destroy_job(ctx, J);
  return OIDT_OK;
}

int32_t oidt_job_reset(oidt_ctx *ctx, uint64_t job) {
  if (!ctx) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  CU(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  CU(ctx, cudaStreamWaitEvent(st, J->ready, 0));
  const JobPlan &pl = J->pl;
  for (int b = 0; b < pl.nbuf; ++b)
    for (int f : fields_of(J->d.mode)) CU(ctx, cudaMemsetAsync(J->mem + pl.off_f[b][f], 0, pl.N * pl.esz, st));
  for (auto fa : psi_pairs(J->d.mode))
    for (int b = 0; b < psi_bufs(pl.nbuf, pl.variant, fa.first); ++b)
      for (int sd = 0; sd < 2; ++sd)
        CU(ctx, cudaMemsetAsync(J->mem + pl.off_psi[b][fa.first][fa.second][sd], 0,
                                psi_elems(J->d.mode, fa.second, J->d.nx, J->d.ny, J->d.nz, J->d.num_cpml,
                                          pl.psi_pitch, pl.psz) * pl.esz, st));
  CU(ctx, cudaMemsetAsync(J->mem + pl.off_ring, 0, pl.off_acc - pl.off_ring, st));
  CU(ctx, cudaMemsetAsync(J->mem + pl.off_acc, 0, pl.off_state - pl.off_acc, st));
  CU(ctx, cudaMemsetAsync(J->mem + pl.off_state, 0, 64, st));
  if (pl.probe_bytes) CU(ctx, cudaMemsetAsync(J->mem + pl.off_probe, 0, pl.probe_bytes, st));
  if (pl.variant == kVariantWave)  // the ordered form's counters restart with the steps
    CU(ctx, cudaMemsetAsync(J->mem + pl.off_wave, 0, 8 + (size_t)4 * (J->d.ie - J->d.ib), st));
  if (pl.variant == kVariantTile)  // the tiles' sub-block counters: equal (zero) again
    CU(ctx, cudaMemsetAsync(J->mem + pl.off_tile, 0, (size_t)4 * kTileMaxBlocks, st));
  CU(ctx, cudaEventRecord(J->done, st));
  J->busy = true;
  J->steps_enqueued = 0;
  J->parity = 0;
  return OIDT_OK;
}

int32_t oidt_job_set_wait_limit(oidt_ctx *ctx, uint64_t job, int64_t cycles) {
  if (!ctx) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  CU(ctx, cudaSetDevice(ctx->device));
  CU(ctx, cudaEventSynchronize(J->done));  // no launch holds the old parameters
  J->wait_cycles = cycles > 0 ? (long long)cycles : kWaitCycles;
  for (int b = 0; b < 2; ++b) {
    J->pvf[b].wait_cycles = J->pcf[b].wait_cycles = J->wait_cycles;
    J->pvd[b].wait_cycles = J->pcd[b].wait_cycles = J->wait_cycles;
    if (J->graph[b]) {  // captured with the old parameters: capture again at next use
      cudaGraphExecDestroy(J->graph[b]);
      J->graph[b] = nullptr;
    }
  }
  return OIDT_OK;
}

int32_t oidt_ctx_stream(oidt_ctx *ctx, void **stream) {
  if (!ctx || !stream) return OIDT_ERR_INVALID;
  *stream = (void *)ctx->stream;
  return OIDT_OK;
}

int32_t oidt_job_profile(oidt_ctx *ctx, uint64_t job, int32_t nsteps, float *ms_out) {
  if (!ctx || !ms_out || nsteps <= 0) return OIDT_ERR_INVALID;
  std::lock_guard<std::mutex> g(ctx->mu);
  Job *J = find(ctx, job);
  if (!J) return fail(ctx, OIDT_ERR_NOTFOUND, "unknown job %llu", (unsigned long long)job);
  if (nsteps > J->pl.K) return fail(ctx, OIDT_ERR_INVALID, "profile at most ring_steps (%d) steps", J->pl.K);
  if (J->steps_enqueued + nsteps > J->d.nt) return fail(ctx, OIDT_ERR_STATE, "not enough source steps left");
  CU(ctx, cudaSetDevice(ctx->device));
  const bool f64 = J->d.precision == OIDT_F64, ex = J->d.arith == OIDT_ARITH_EXACT;
  if (f64) return ex ? profile_t<double, true>(ctx, J, nsteps, ms_out) : profile_t<double, false>(ctx, J, nsteps, ms_out);
  return ex ? profile_t<float, true>(ctx, J, nsteps, ms_out) : profile_t<float, false>(ctx, J, nsteps, ms_out);
}

}  // extern "C"
