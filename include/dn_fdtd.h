/*
 * dn_fdtd.h -- C ABI of the B200 (sm_100a) Yee-FDTD library (libdn_fdtd.so).
 *
 * Plain C: raw device pointers, sizes and strides, int status codes, no C++
 * exceptions and no torch types cross this boundary.  All buffers are owned
 * by the caller (the Python layer allocates them with PyTorch); every call is
 * asynchronous on the given CUDA stream (passed as `void*`, a cudaStream_t;
 * NULL = legacy default stream) unless its comment says otherwise.
 *
 * Layout: a field is a (D, H, W) array, W (x, index k) fastest, then H (y,
 * index j), then D (z, index i).  Rows are `pitch_y` elements apart and
 * planes `pitch_z` elements apart; for the 3-D kernels pitch_y * element size
 * must be a multiple of 16 bytes and every field base 16-byte aligned (the
 * Python layer pads rows to 32 elements).  2-D grids use D = 1, index (j, k)
 * = (row, column) and ignore pitch_z.
 *
 * Reference interfaces replaced (DiffNano, paths relative to its checkout):
 *   dn_fdtd2d_run  <- FDTDSolver2D._run_steps loop body: _time_step_tm /
 *                     _time_step_te + `field + mask*waveform`
 *                     (diffnano/solvers/fdtd2d.py:233-303, 330-357)
 *   dn_fdtd3d_run  <- FDTDSolver3D._run_steps loop body: _time_step +
 *                     `Ez + mask*waveform` (diffnano/solvers/fdtd3d.py:378-465,
 *                     490-502)
 */
#ifndef DN_FDTD_H
#define DN_FDTD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DN_OK            0
#define DN_EINVAL        1  /* bad argument (shape, pointer, alignment, size) */
#define DN_ENOMEM        2  /* a limit of a fixed-size resource was exceeded   */
#define DN_ECUDA         3  /* a CUDA runtime/driver call failed               */
#define DN_ETIMEOUT      4  /* a bounded device-side wait gave up              */
#define DN_ENONFINITE    5  /* a NaN/Inf was detected                          */
#define DN_EUNSUPPORTED  6  /* no kernel for this configuration / device       */

/* ---- enums ------------------------------------------------------------- */
#define DN_F32 0
#define DN_F64 1

/* field components; also the index into the 6-pointer field sets */
#define DN_EX 0
#define DN_EY 1
#define DN_EZ 2
#define DN_HX 3
#define DN_HY 4
#define DN_HZ 5
#define DN_NONE (-1)

/* 2-D polarisations */
#define DN_TM 0 /* Ez, Hx, Hy  (fdtd2d.py:233-267) */
#define DN_TE 1 /* Hz, Ex, Ey  (fdtd2d.py:269-303) */

/* 3-D CPML axis mapping */
#define DN_AXES_REFERENCE 0 /* the reference's broadcasting (fdtd3d.py:402-463); cubic grids */
#define DN_AXES_PHYSICAL  1 /* every profile indexed along its own axis; any (D, H, W)       */

#define DN_MAX_MONITORS 4
#define DN_MAX_FREQS 16

/* half-open index box, axis order (z, y, x); 2-D uses z = [0, 1) */
typedef struct {
  int32_t lo[3];
  int32_t hi[3];
} dn_box;

typedef struct {
  int32_t D, H, W;
  int32_t dtype;   /* DN_F32 / DN_F64: element type of fields, coefficients, wave table */
  int64_t pitch_y; /* elements between rows   (>= W)         */
  int64_t pitch_z; /* elements between planes (>= H*pitch_y) */
  double dt;       /* time step (c = 1, nm units)            */
  double dl;       /* cell size (nm)                         */
  int32_t axes;    /* 3-D only: DN_AXES_*                     */
  int32_t pol;     /* 2-D only: DN_TM / DN_TE                 */
} dn_grid;

/* CPML profiles (FP64, device): index 0 = z (length D), 1 = y (H), 2 = x (W).
 * b = exp(-(s+a)dt), c = s(b-1)/(s+a) as in fdtd2d.py:67-88.  2-D uses y, x. */
typedef struct {
  const double* b[3];
  const double* c[3];
} dn_cpml;

/* soft source: after each full step, field[component][box] += wave[t]
 * (fdtd2d.py:333,351; fdtd3d.py:502).  `wave` is indexed by the absolute
 * step t, has the grid's dtype and holds `n_t` entries: a run of steps
 * t0 .. t0+nsteps-1 needs t0 + nsteps <= n_t (DN_EINVAL otherwise).
 * component = DN_NONE disables it. */
typedef struct {
  int32_t component;
  dn_box box;
  const void* wave;
  int32_t n_t;
} dn_source;

/* running-DFT monitor (extension, no reference counterpart):
 * acc[f][cell][0..1] += v_t(cell) * phase[t][f][0..1] on every step t, where
 * v_t is the component's value after step t (source included) and
 * phase[t][f] = (cos(w_f t dt) dt, -sin(w_f t dt) dt).  Cells are the box's
 * cells in (z, y, x) row-major order.  FP64 accumulators.  `phase` has n_t
 * rows (absolute steps 0 .. n_t-1): every step a forward run or a reverse
 * sweep touches must be below n_t (DN_EINVAL otherwise). */
typedef struct {
  int32_t component;
  dn_box box;
  int32_t n_freq;
  const double* phase; /* [n_t][n_freq][2] device */
  double* acc;         /* [n_freq][cells][2] device, caller zeroes it */
  int32_t n_t;
} dn_monitor;

/* single-cell probe (fdtd2d.py:335-337 snapshots, fdtd3d.py:698 time_series):
 * out[t] = value of `component` at (pos[0], pos[1], pos[2]) = (z, y, x) after
 * step t (source included).  `out` has the grid dtype, is indexed by the
 * absolute step t and holds `n_t` entries (t0 + nsteps <= n_t, DN_EINVAL
 * otherwise).  component = DN_NONE disables it. */
typedef struct {
  int32_t component;
  int32_t pos[3];
  void* out;
  int32_t n_t;
} dn_probe;

/* curl record (forward replay for the adjoint): during step t the bracket
 * term of each eps-dependent update -- the part multiplied by dt/eps -- is
 * stored at curl[c] + (t - t0) * step_stride + cell (cell = the field layout
 * offset), for t0 <= t < t0 + nslots.  3-D records Ex, Ey, Ez (curl[0..2]);
 * 2-D TM records Ez in curl[2]; 2-D TE records Ex, Ey in curl[0], curl[1].
 * Grid dtype. */
typedef struct {
  void* curl[3];
  int64_t step_stride;
  int32_t t0;
  int32_t nslots;
} dn_curl_record;

/* ---- library information ------------------------------------------------ */
const char* dn_strerror(int32_t status);
/* sizeof of an ABI struct by name ("dn_grid", "dn_batch2d_inst", ...), -1 if
 * unknown: lets a binding check its struct mirrors */
int64_t dn_struct_size(const char* name);
int32_t dn_version(void);
/* last CUDA error code seen by the library on this thread (0 if none) */
int32_t dn_last_cuda_error(void);

/* ---- forward time stepping --------------------------------------------- */
/*
 * Run `nsteps` leapfrog steps t = t0 .. t0+nsteps-1 of the 2-D TM/TE solver.
 * Fields ping-pong: step t reads set `fa` when (t - t0) is even and writes
 * `fb`, and the reverse when odd; *final_in_b tells where the result is.
 * Field sets are 6 pointers indexed by DN_EX..DN_HZ; only the polarisation's
 * three are used.  `ce` is the per-cell coefficient dt/eps_r (grid dtype,
 * same layout as the fields).  `src`, `mons` and `probe` may be NULL.  `status`
 * (device int32, may be NULL) receives device-side error codes and is never
 * cleared by the library.
 */
int32_t dn_fdtd2d_run(const dn_grid* g, void* const fa[6], void* const fb[6], const void* ce,
                      const dn_cpml* cpml, const dn_source* src, const dn_monitor* mons,
                      int32_t n_mon, const dn_probe* probe, const dn_curl_record* rec,
                      int32_t t0, int32_t nsteps, int32_t* status, void* stream,
                      int32_t* final_in_b);

/* 3-D analogue (all six components), same ping-pong and status contract.
 * Field bases and ce must be 16-byte aligned, pitches multiples of 16 bytes. */
int32_t dn_fdtd3d_run(const dn_grid* g, void* const fa[6], void* const fb[6], const void* ce,
                      const dn_cpml* cpml, const dn_source* src, const dn_monitor* mons,
                      int32_t n_mon, const dn_probe* probe, const dn_curl_record* rec,
                      int32_t t0, int32_t nsteps, int32_t* status, void* stream,
                      int32_t* final_in_b);

/* ---- adjoint (reverse) time stepping ------------------------------------
 * Discrete adjoint of the steps above: runs reverse steps t = t_end-1 down
 * to t_end-nsteps.  `la`/`lb` are 6-pointer sets of adjoint fields (the
 * gradient of the loss with respect to each field after step t), ping-pong
 * like the forward; on entry `la` holds the adjoint after step t_end-1.
 * `curl` is the record of a forward replay covering those steps (see
 * dn_curl_record).  `grad_ce` (FP64, field layout) accumulates
 * dL/d(dt/eps) = sum_t lambda_E(t) . curl(t).  `mons` carry, in `acc`, the
 * gradient of the loss with respect to each monitor's DFT (re, im); they are
 * injected into the adjoint field before each reverse step.  The source term
 * does not depend on eps and has no adjoint.
 * Replaces the reference's backward passes: autograd through
 * _time_step (diffnano/solvers/fdtd3d.py:378-465, fdtd2d.py:233-303) and
 * _TimeReversalFDTD.backward (fdtd3d.py:166-219). */
int32_t dn_fdtd2d_adjoint(const dn_grid* g, void* const la[6], void* const lb[6], const void* ce,
                          const dn_cpml* cpml, const dn_curl_record* curl, double* grad_ce,
                          const dn_monitor* mons, int32_t n_mon, int32_t t_end, int32_t nsteps,
                          int32_t* status, void* stream, int32_t* final_in_b);
int32_t dn_fdtd3d_adjoint(const dn_grid* g, void* const la[6], void* const lb[6], const void* ce,
                          const dn_cpml* cpml, const dn_curl_record* curl, double* grad_ce,
                          const dn_monitor* mons, int32_t n_mon, int32_t t_end, int32_t nsteps,
                          int32_t* status, void* stream, int32_t* final_in_b);

/* ---- batched 2-D instances in one persistent launch ----------------------
 * Many independent 2-D grids of different sizes and step counts (robust-
 * design variants, wavelength sweeps) advanced together by one persistent
 * cooperative kernel: each global step processes every tile of every
 * instance that still has steps left, then all CTAs meet at a grid barrier
 * (bounded spin; DN_ETIMEOUT on expiry).  The backward kernel walks the
 * checkpoint segments from the last: it replays each segment from its
 * checkpoint with the curl record on, then runs the segment's reverse steps,
 * injecting monitor-DFT gradients as it loads the adjoint field.
 * No reference counterpart (the reference runs one solver object per grid).
 *
 * Per instance (host array, packed by dn_batch2d_pack into a device table):
 * fields are the polarisation's three components in the order TM (Ez, Hx,
 * Hy) / TE (Hz, Ex, Ey), each H x pitch elements, two ping-pong sets; after
 * n_steps the state is in set n_steps % 2.  Checkpoints (states at steps K,
 * 2K, ... < n_steps) are [slot-1][3][H*pitch]; the curl record of one segment
 * is [K][ncurl][H*pitch] (TM: Ez; TE: Ex, Ey); adjoint sets likewise, the
 * gradient of the final field goes into lam[n_steps % 2] before the backward
 * launch, the result accumulates into grad (FP64 [H*pitch]).  Rows move in
 * 16-byte chunks: pitch * element size (and pitch * 8, for grad) must be a
 * multiple of 16 bytes and every array 16-byte aligned (DN_EINVAL otherwise). */
typedef struct {
  int32_t H, W;
  int64_t pitch;
  int32_t n_steps;
  int32_t src_comp;           /* DN_EZ (TM) / DN_HZ (TE) / DN_NONE */
  dn_box src_box;
  const void* wave;           /* [n_steps] */
  void* f[2][3];
  const void* ce;
  const double* b[2];         /* CPML: [0] rows (length H), [1] columns (length W) */
  const double* c[2];
  double dt, dl;
  int32_t mon_comp;           /* DN_NONE or the polarisation's first field */
  dn_box mon_box;
  int32_t n_freq;
  const double* phase;        /* [n_steps][n_freq][2] */
  double* acc;                /* [n_freq][cells][2] */
  void* ckpt;
  void* curl;
  void* lam[2][3];
  double* grad;
  const double* gmon;         /* [n_freq][cells][2], may be NULL */
} dn_batch2d_inst;

typedef struct {
  int32_t pol;        /* DN_TM / DN_TE, all instances */
  int32_t dtype;      /* DN_F32 / DN_F64 */
  int32_t n_inst;
  int32_t K;          /* checkpoint interval in steps (>= 1) */
  int32_t tile_rows;  /* 8, 16 or 32 (tile = tile_rows x 128 cells in FP32, x 64 in FP64;
                         each of its 8 warps marches tile_rows / 8 rows) */
  int32_t max_ctas;   /* upper bound on the persistent grid (0: as many as fit) */
} dn_batch2d;

/* bytes of the device table for this batch */
int64_t dn_batch2d_table_bytes(const dn_batch2d* cfg, const dn_batch2d_inst* insts);
/* pack the batch into `host_table` (dn_batch2d_table_bytes bytes); the caller
 * copies it to device memory and passes that copy to the launches below */
int32_t dn_batch2d_pack(const dn_batch2d* cfg, const dn_batch2d_inst* insts, void* host_table,
                        int64_t bytes);
/* forward: all steps of all instances (monitors accumulate, checkpoints are
 * written when K < n_steps) in one persistent launch */
int32_t dn_batch2d_forward(const dn_batch2d* cfg, void* dev_table, int32_t* status,
                           void* stream);
/* backward: replay + reverse sweep of all instances in one persistent launch */
int32_t dn_batch2d_backward(const dn_batch2d* cfg, void* dev_table, int32_t* status,
                            void* stream);

/* Forward-only solve of every instance of a packed table with each grid held
 * in the shared memory of one thread-block cluster (CTAs own row bands, the
 * neighbouring rows come from the next / previous CTA's shared memory): no
 * global traffic for the fields between the first and the last step.  Same
 * results as dn_batch2d_forward (final fields in f[n_steps % 2], monitor DFTs
 * accumulated), no checkpoints.  Where the grid fits twice, the fields are
 * double-buffered and each step takes one cluster barrier (the neighbour row
 * of the second half-step is recomputed locally); otherwise they are updated
 * in place with two barriers per step.
 * dn_batch2d_cluster_size returns the value to pass as `cluster`: the cluster
 * size (16, else 8 CTAs per grid), with DN_CLUSTER_DOUBLE_BUFFERED set for the
 * double-buffered kernel, and sets *smem_bytes (per CTA); 0 when some instance
 * is too large for a cluster, -1 on invalid input. */
#define DN_CLUSTER_DOUBLE_BUFFERED 0x100
int32_t dn_batch2d_cluster_size(const dn_batch2d* cfg, const dn_batch2d_inst* insts,
                                int64_t* smem_bytes);
int32_t dn_batch2d_forward_cluster(const dn_batch2d* cfg, void* dev_table, int32_t cluster,
                                   int64_t smem_bytes, void* stream);

/* Diagnostic, no reference counterpart: runs the persistent kernels' grid
 * barrier alone, `rounds` times, on `n_ctas` one-warp CTAs (at most one per
 * SM), waiting for n_ctas + `missing` arrivals with at most `spin_limit`
 * probes 64 ns apart (1 .. 2^24, the kernels' own limit).  missing = 0 must
 * leave *status at DN_OK; missing > 0 arrivals never come, so every CTA's wait
 * runs out and *status becomes DN_ETIMEOUT (the launch returns, the context
 * stays usable).  `dev_bar`: 16 bytes of device memory, 16-byte aligned,
 * cleared by the call; `status`: a device int32 the caller zeroes. */
int32_t dn_batch2d_barrier_selftest(int32_t n_ctas, int32_t missing, int64_t spin_limit,
                                    int32_t rounds, void* dev_bar, int32_t* status,
                                    void* stream);

/* ---- figure of merit ----------------------------------------------------
 * *out = sum_i |dft[i]|^2 over n_complex FP64 (re, im) pairs, reduced in FP64
 * (warp-shuffle trees, per-block partials in `scratch`, deterministic final
 * sum).  No reference counterpart (the reference has no monitors); it is the
 * FOM of the design workloads (sum of |DFT E|^2 over a monitor).  `scratch`
 * needs dn_fom_abs2_scratch_bytes(n_complex) bytes, 16-byte aligned. */
int64_t dn_fom_abs2_scratch_bytes(int64_t n_complex);
int32_t dn_fom_abs2(const double* dft, int64_t n_complex, double* out, void* scratch,
                    int64_t scratch_bytes, void* stream);

/* ---- non-finite watchdog -------------------------------------------------
 * No reference counterpart: the reference returns NaN fields and gradients
 * without an error (its TE update grows exponentially and overflows FP32
 * within a few hundred steps, diffnano/solvers/fdtd2d.py:269-303).  Scans
 * `n_spans` (1 .. DN_MAX_SPANS) strided device arrays and, when any element
 * is NaN or +-Inf, records DN_ENONFINITE in the device word *status if it
 * still holds DN_OK.  NaN and Inf are sticky under the leapfrog update, so a
 * scan of a solve's final fields, monitor DFTs and gradient catches a blow-up
 * at any step; the solvers do it once per solve and per reverse sweep. */
typedef struct {
  const void* ptr;
  int32_t dtype;  /* DN_F32 / DN_F64 */
  int64_t rows;   /* rows of `cols` elements ...                    */
  int64_t cols;
  int64_t pitch;  /* ... `pitch` elements apart (pitch >= cols)     */
} dn_span;
#define DN_MAX_SPANS 32
int32_t dn_check_finite(const dn_span* spans, int32_t n_spans, int32_t* status, void* stream);

/* ---- stepping without device allocation --------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory where they step the solver (a plugin inside an application that owns
 * the whole device-memory budget, a loop whose policy forbids allocation):
 * dn_fdtd2d_run with the second ping-pong set replaced by a file-scope device
 * array of DN_NOALLOC_MAX_BYTES held by every GPU that loads the library.
 * `f` (6 pointers, the polarisation's three used) is read and updated in
 * place; the result is always in `f`.  Grids needing more than
 * DN_NOALLOC_MAX_BYTES for three fields (H * pitch_y * element size each,
 * rounded up to 256 bytes) return DN_ENOMEM.  The first call on a device
 * looks up the array's address; make it before any stream capture.  The
 * address stays cached for the process: after cudaDeviceReset on a device,
 * do not call this entry point on that device again.  All calls share the
 * array: calls whose GPU work overlaps race.  Makes no cudaMalloc/cudaFree
 * or other allocating call. */
#define DN_NOALLOC_MAX_BYTES (6 * 1024 * 1024)
int32_t dn_fdtd2d_run_noalloc(const dn_grid* g, void* const f[6], const void* ce,
                              const dn_cpml* cpml, const dn_source* src, const dn_monitor* mons,
                              int32_t n_mon, const dn_probe* probe, int32_t t0, int32_t nsteps,
                              int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DN_FDTD_H */
