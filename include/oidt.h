/*
 * oidt.h -- C ABI of liboidt.so, the B200 (sm_100a) FDTD S-parameter engine.
 *
 * The reference runs one simulation per process: its fdtd_main.py builds the
 * grid, copies every array to the device once
 * (FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_main.py:216-261), launches
 * 12 (2D) or 23 (3D) Numba kernels per time step (fdtd_main.py:275-304;
 * FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_main.py:357-406) and copies the
 * port DFT accumulators back (fdtd_main.py:349-357).  This ABI replaces that
 * device boundary with a job API: a job owns all device state of one
 * simulation; host buffers are only borrowed for the duration of a call.
 *
 * Conventions
 *  - Every function returns 0 (OIDT_OK) or a negative OIDT_ERR_* code; the
 *    message is available from oidt_last_error(ctx).  No C++ exception
 *    crosses this boundary.
 *  - Arrays use the reference layout: 2D [nx][ny], 3D [nx][ny][nz], C order,
 *    element type given by oidt_job_desc.precision.
 *  - Field ids: OIDT_EX..OIDT_HZ.  2D TM uses EZ, HX, HY; 2D TE uses EX, EY,
 *    HZ (the reference's fdtd_funcs.py kernels of each solver).
 *  - Waits are bounded: oidt_job_sync returns OIDT_ERR_TIMEOUT after
 *    timeout_ms instead of blocking forever.
 */
#ifndef OIDT_H
#define OIDT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OIDT_ABI_VERSION 5  /* 2: line probe (oidt_job_desc.probe, oidt_job_read_probe);
                              3: launch choices (reserved[2..3]), oidt_job_port_power;
                              4: oidt_job_read_dft_window_static, the vector and ordered
                                 launch forms (reserved[0] = 2, 3), oidt_job_set_wait_limit,
                                 the material index (mat_idx, mat_tab, nmat);
                              5: the 2D tile form (reserved[0] = 4 in 2D, its choices in
                                 reserved[2..3]); 2D jobs take launch forms 0 and 4 only */

/* status codes */
#define OIDT_OK 0
#define OIDT_ERR_INVALID (-1)  /* bad argument or descriptor            */
#define OIDT_ERR_CUDA (-2)     /* CUDA runtime error                      */
#define OIDT_ERR_BUDGET (-3)   /* admission would exceed the HBM budget   */
#define OIDT_ERR_NOTFOUND (-4) /* unknown job id                          */
#define OIDT_ERR_TIMEOUT (-5)  /* bounded wait expired                    */
#define OIDT_ERR_STATE (-6)    /* call not valid in the job's state       */

/* solvers: the three reference directories FDTD/GPU/FDTD_{2D_TM,2D_TE,3D} */
#define OIDT_MODE_TM2 0
#define OIDT_MODE_TE2 1
#define OIDT_MODE_YEE3D 2

#define OIDT_F32 0
#define OIDT_F64 1

/* OIDT_ARITH_FAST: reciprocal multiplies and fused multiply-adds.
 * OIDT_ARITH_EXACT: the reference's operation order with IEEE divisions and
 * no contraction, so a float64 run reproduces the reference's float64 run
 * bit for bit. */
#define OIDT_ARITH_FAST 0
#define OIDT_ARITH_EXACT 1

#define OIDT_EX 0
#define OIDT_EY 1
#define OIDT_EZ 2
#define OIDT_HX 3
#define OIDT_HY 4
#define OIDT_HZ 5

typedef struct oidt_ctx oidt_ctx;

/* One simulation.  Mirrors the arrays and scalars the reference passes to
 * its kernels (fdtd_main.py:216-261, 3D :258-343). */
typedef struct oidt_job_desc {
  int32_t mode;      /* OIDT_MODE_*                                        */
  int32_t precision; /* OIDT_F32 / OIDT_F64: fields, coefficients, psi     */
  int32_t arith;     /* OIDT_ARITH_*                                       */
  int32_t nx, ny, nz;/* nz = 1 in 2D                                       */
  int32_t num_cpml;  /* P                                                  */
  int32_t ib, jb, kb, ie, je, ke; /* update limits (reference offset = 2)  */
  int32_t nt;        /* steps covered by j_src and the twiddle tables      */
  int32_t nf;        /* DFT frequencies                                    */
  /* E-component update coefficients dt/eps, full grids:
   * TM2 {CBZ}, TE2 {CBX, CBY}, 3D {CBX, CBY, CBZ}; unused entries NULL */
  const void *cb[3];
  /* kappa*dx divisors: kxe, kye, kze, kxh, kyh, kzh (length nx, ny, nz);
   * 2D: kze = kzh = NULL */
  const void *kdx[6];
  const void *be, *ce, *bh, *ch; /* CPML recursion coefficients [P]        */
  double db;         /* dt/mu, cast to precision                           */
  double dx;         /* the divisor the CPML kernels use                   */
  /* soft source: field[src_lo..src_hi) -= j_src[n] each step              */
  int32_t src_field;
  int32_t src_lo[3], src_hi[3];
  const void *j_src; /* [nt]                                               */
  /* port DFT planes: 2D x = port_pos[q], window j in [win_lo[1], win_hi[1]);
   * 3D z = port_pos[q], window i in [win_lo[0], win_hi[0]), j in
   * [win_lo[1], win_hi[1]) */
  int32_t port_pos[2];
  int32_t win_lo[2], win_hi[2];
  /* float64 twiddles [nf][nt]: cos/sin(2 pi f n dt) and at (n + 1/2) dt */
  const double *cos_e, *sin_e, *cos_h, *sin_h;
  int32_t ring_steps; /* steps buffered between DFT folds (0 = default)    */
  /* reserved[0]: launch form.  3D: 0 = per-cell E-half / H-half launches,
   *              1 = plane sweep (one launch per step),
   *              2 = vector form: the E-half / H-half launches with four
   *                  cells per thread along z and 16-byte accesses,
   *              3 = ordered form: the vector form's code in one launch per
   *                  step, E and H half-steps ordered plane by plane.
   *              2D: 0 = per-cell E-half / H-half launches,
   *              4 = tile form: each block advances a tile of the grid and a
   *                  halo around it through sub-blocks of up to 8 steps in
   *                  shared memory; a ring block is one cooperative launch
   *                  where every tile is resident at once;
   * reserved[1]: 1 = launch every step directly (no CUDA-graph replay);
   * reserved[2]: 3D per-cell form: rows of a block's 32 x rows tile,
   *              2, 4 or 8 (0 = 4); 2D tile form: 1 = one launch per
   *              sub-block instead of the cooperative launch;
   * reserved[3]: 3D plane sweep: march depth, the x-planes of one work item
   *              (0 = the engine's makespan estimate); 2D tile form: steps
   *              per sub-block, 1 to 8 (0 = the engine's estimate).
   * None of these changes results; they are launch choices, measured per
   * grid shape by the host's tuner.  Other values are OIDT_ERR_INVALID. */
  int32_t reserved[4];
  /* 3D time-domain line probe, the wave-impedance runs' recording
   * (FDTD/GPU/FDTD_3D/wave_impedance/fdtd_main.py:298-299, fdtd_funcs.py:
   * map_efield_zwave / map_hfield_zwave): probe[0] = 1 records after every
   * step, for x in [0, ie), Ey(x, y, z) averaged over y, y+1; Ez averaged over
   * z, z+1; Hy over (x, x+1) x (z, z+1); Hz over (x, x+1) x (y, y+1), at
   * y = probe[1], z = probe[2].  probe[0] = 0: no probe (probe[1..2] 0). */
  int32_t probe[3];
  /* 3D only, optional: the dt/eps grids as a material index.  With mat_idx
   * != NULL every cell's (CBX, CBY, CBZ) is mat_tab[mat_idx[cell]]:
   * mat_idx [nx][ny][nz] bytes (C order), mat_tab [nmat][3] values in the
   * job's precision, 1 <= nmat <= 256; cb[] is not read (NULL allowed).  The
   * engine expands the grids on the device for the forms that read them; the
   * vector form reads the index (1 byte per cell instead of three values).
   * Results equal those of the expanded grids passed in cb[].  NULL: none
   * (nmat 0).  No counterpart in the reference, whose CB arrays are built
   * from its foreground mask (fdtd_main.py:86-118 (3D)). */
  const uint8_t *mat_idx;
  const void *mat_tab;
  int32_t nmat;
} oidt_job_desc;

typedef struct oidt_stats {
  uint64_t hbm_budget;   /* admission budget in bytes                      */
  uint64_t hbm_in_use;   /* bytes held by live jobs                        */
  int32_t live_jobs;
  int32_t device;
  int64_t kernel_launches; /* kernels this context has launched            */
} oidt_stats;

int32_t oidt_abi_version(void);

/* Context: one per device.  hbm_budget = 0 means 90 % of free memory. */
int32_t oidt_create(int32_t device, uint64_t hbm_budget, oidt_ctx **out);
int32_t oidt_destroy(oidt_ctx *ctx);
const char *oidt_last_error(oidt_ctx *ctx);
int32_t oidt_stats_get(oidt_ctx *ctx, oidt_stats *out);

/* Device bytes a job with this descriptor would hold (admission check). */
int32_t oidt_job_bytes(const oidt_job_desc *desc, uint64_t *bytes);

/* Allocate device state, copy the descriptor's host arrays (H2D), zero the
 * fields, psi and DFT accumulators.  Replaces fdtd_main.py:51-261. */
int32_t oidt_job_create(oidt_ctx *ctx, const oidt_job_desc *desc, uint64_t *job);

/* Enqueue nsteps time steps (asynchronous).  Replaces the hot loop
 * fdtd_main.py:275-304 (3D :357-406); the DFT fold runs every ring_steps
 * steps and at the end of the call. */
int32_t oidt_job_advance(oidt_ctx *ctx, uint64_t job, int32_t nsteps);

/* Advance several jobs together (they may differ in size and solver; they
 * must share ring_steps): every ring block of steps forks one branch per job
 * onto auxiliary streams, so independent jobs run concurrently.  A job's full
 * ring block is its own CUDA graph (captured at its first full block, the
 * graph oidt_job_advance replays), so a group whose membership changes from
 * call to call costs no capture. */
int32_t oidt_batch_advance(oidt_ctx *ctx, const uint64_t *jobs, int32_t njobs, int32_t nsteps);

/* Bounded wait for the job's enqueued work.  timeout_ms < 0: no limit. */
int32_t oidt_job_sync(oidt_ctx *ctx, uint64_t job, int32_t timeout_ms);

/* Steps completed so far (after a sync) and whether work is in flight. */
int32_t oidt_job_query(oidt_ctx *ctx, uint64_t job, int32_t *steps_done, int32_t *busy);

/* Port DFT of one component as complex128 (re, im interleaved), reference
 * layout: 2D [nf][ny], 3D [nf][nx][ny], zero outside the window.
 * comp: 2D 0 = E (Ez TM / Ey TE), 1 = H (Hy TM / Hz TE);
 *       3D 0 = Ex, 1 = Ey, 2 = Hx, 3 = Hy.  Replaces fdtd_main.py:349-363. */
int32_t oidt_job_read_dft(oidt_ctx *ctx, uint64_t job, int32_t port, int32_t comp,
                          double *out_re_im, size_t n_doubles);

/* Line-probe record of one component as [nt][nx] elements of the job's
 * precision (rows of steps not yet run are 0).  comp: 0 = Ey, 1 = Ez,
 * 2 = Hy, 3 = Hz.  Replaces the wave-impedance runs' copy of their
 * [nt, nx] recordings (FDTD/GPU/FDTD_3D/wave_impedance/fdtd_main.py:341-346).
 * OIDT_ERR_STATE if the job has no probe. */
int32_t oidt_job_read_probe(oidt_ctx *ctx, uint64_t job, int32_t comp, void *out, size_t nbytes);

/* Complex power through one port's plane, summed over a window on the
 * device in float64: out[f] = sum over the window of the Poynting density
 * 3D 1/2 (Ex Hy* - Ey Hx*), 2D TM -1/2 Ez Hy*, 2D TE 1/2 Ey Hz*, of this
 * job's port DFT, or, with minus_job != 0, of this job's minus minus_job's
 * at the same port (the reflected wave: device-under-test run minus
 * incident run; same mode, nf and port plane required).  These are the sums
 * S_ij = sqrt(P_ref / P_inc) is formed from (FDTD/GPU/FDTD_2D_TM/
 * s-parameter_extraction/extract_sparams.py:88-104, FDTD_3D/.../
 * extract_sparams.py:114-131, which sum over the window on the host after
 * the [nf, plane] arrays were saved and loaded); here only nf complex
 * values cross the link.  window = {i0, i1, j0, j1}: rows [i0, i1) x columns [j0, j1)
 * of the port plane, 3D [nx][ny], 2D one row of ny (i0 = 0, i1 = 1).
 * out = nf complex128 (re, im interleaved; n_doubles >= 2 nf).  Waits for
 * the steps enqueued on both jobs, on a stream of its own.  The summation
 * order is fixed (block tree per frequency), so results are deterministic;
 * they equal the host sums up to float64 rounding. */
int32_t oidt_job_port_power(oidt_ctx *ctx, uint64_t job, uint64_t minus_job, int32_t port,
                            const int32_t window[4], double *out_re_im, size_t n_doubles);

/* Port-window DFT of one (port, comp), as oidt_job_read_dft but restricted
 * to the DFT window [win_lo, win_hi): out = complex128 [nf][wi][wj] (3D, wi =
 * win_hi[0] - win_lo[0], wj = win_hi[1] - win_lo[1]) or [nf][wj] (2D),
 * interleaved re/im, n = number of doubles.  Allocates nothing, for hosts
 * that may not allocate device memory where they read results: a host that
 * reserves its whole device budget at start-up (a fixed-budget serving
 * process) or reads results from a callback where an allocation could
 * block on, or fail under, memory held by others.  It stages through a fixed
 * 16 MiB static device buffer, held on every GPU that loads the library
 * until the process exits; windows needing more are rejected with
 * OIDT_ERR_INVALID.  Nothing in the buffer has to start at zero: every
 * element read was written by the same call.  The first call on a device
 * resolves the buffer's address (cudaGetSymbolAddress, which may load the
 * module) and should come before any stream capture on that device.  All
 * contexts on a device share the buffer, which keeps the last call's
 * contents: calls that overlap on one device race.  No counterpart in the
 * reference (its DFT arrays come back whole, fdtd_main.py:349-386). */
int32_t oidt_job_read_dft_window_static(oidt_ctx *ctx, uint64_t job, int32_t port, int32_t comp,
                                        double *out, size_t n);

/* Field snapshot / overwrite (reference layout, job precision). */
int32_t oidt_job_read_field(oidt_ctx *ctx, uint64_t job, int32_t field, void *out, size_t nbytes);
int32_t oidt_job_write_field(oidt_ctx *ctx, uint64_t job, int32_t field, const void *src, size_t nbytes);

/* CPML auxiliary array of field `field` for slab axis `axis` (0 x, 1 y, 2 z)
 * and side (0 low, 1 high), in the reference's PSI_<F>_<A><LO|HI> layout. */
int32_t oidt_job_read_psi(oidt_ctx *ctx, uint64_t job, int32_t field, int32_t axis, int32_t side,
                          void *out, size_t nbytes);

int32_t oidt_job_release(oidt_ctx *ctx, uint64_t job);

/* Return the job to step 0 (zero fields, psi, capture ring, DFT
 * accumulators) keeping its coefficients resident: the next simulation on the
 * same structure without another host-to-device copy.  The reference has no
 * counterpart (it starts a new process per simulation, fdtd_main.py:51-53). */
int32_t oidt_job_reset(oidt_ctx *ctx, uint64_t job);

/* Bound, in SM clock cycles, on each wait of the plane-sweep kernel
 * (reserved[0] = 1) for a plane's tile loads, and of the 2D tile form's
 * cooperative launch for its neighbour tiles between sub-blocks; cycles <= 0
 * restores the default (4e9, about 2 s).  A wait that runs out marks the job
 * failed -- oidt_job_sync then returns OIDT_ERR_TIMEOUT -- and the kernel
 * still ends: the plane sweep after the copies it has in flight have landed
 * (those waits keep the default bound), the tile form's blocks without
 * waiting again in that launch.  For tests of that failure path: a small
 * bound makes the waits run out on loads or neighbours that are merely in
 * flight.  No counterpart in the reference (its kernels do not wait on one
 * another). */
int32_t oidt_job_set_wait_limit(oidt_ctx *ctx, uint64_t job, int64_t cycles);

/* The context's compute stream (a cudaStream_t), so callers can order their
 * own work or record CUDA events around oidt_job_advance. */
int32_t oidt_ctx_stream(oidt_ctx *ctx, void **stream);

/* Run nsteps steps without graph replay, bracketing every launch with CUDA
 * events on the compute stream; ms_out[0..2] receive the average duration of
 * the E-half, H-half and DFT-fold launches.  Replaces the reference's
 * wall-clock MCells/s print (fdtd_main.py:306-341) with per-kernel device
 * times.  A line probe records these steps too (its launches are not timed). */
int32_t oidt_job_profile(oidt_ctx *ctx, uint64_t job, int32_t nsteps, float *ms_out);

#ifdef __cplusplus
}
#endif
#endif /* OIDT_H */
