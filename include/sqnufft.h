/*
 * sqnufft -- B200-native static structure factor S(q) for sqcalc.
 *
 * C ABI of libsqnufft.so.  Every entry point is extern "C", takes plain
 * pointers and sizes, never exits or traps, and returns an int status
 * (0 = ok, 1 = warning, >1 = error; see SQN_ERR_*).
 *
 * The boundary sits one level above the one sqcalc uses today.  sqcalc's GPU
 * method (src/sqc_gpu.f90:108-362) drives cuFINUFFT through iso_c_binding
 * (src/sqc_cufinufft.f90:183-293): makeplan / setpts / execute / destroy plus
 * raw cudaMalloc / cudaMemcpy, then downloads the whole T x prod(modes) mode
 * cube and does the pair sums and the shell binning on the host
 * (src/sqc_structure_factor.f90:457-643).  Here the library owns the whole
 * frame accumulate: positions in, FP64 shell accumulators out; the mode cube
 * never leaves the GPU.  Each entry point below names the reference interface
 * it replaces.
 *
 * Array layouts are the reference's Fortran arrays in memory order:
 *   cell[9]        a(3,3) column major: cell[3*i + r] = component r of vector a_(i+1)
 *   pos            frame%pos(3, natoms) per frame, frames back to back
 *   partial_num    partial_num(ntypes, ntypes, nq), first index fastest
 *   gnum, gden     flat reciprocal grid of prod(modes) values, index gidx - 1
 */
#ifndef SQNUFFT_H
#define SQNUFFT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SQN_ABI_VERSION 2

/* Status codes.  Values shared with FINUFFT keep FINUFFT's numbering
 * (external/finufft/include/finufft_errors.h:5-31). */
enum {
  SQN_OK = 0,
  SQN_WARN_EPS_TOO_SMALL = 1,       /* = FINUFFT_WARN_EPS_TOO_SMALL */
  SQN_ERR_UPSAMPFAC_TOO_SMALL = 7,  /* = FINUFFT_ERR_UPSAMPFAC_TOO_SMALL */
  SQN_ERR_ALLOC = 11,               /* = FINUFFT_ERR_ALLOC */
  SQN_ERR_CUDA = 15,                /* = FINUFFT_ERR_CUDA_FAILURE */
  SQN_ERR_PLAN_NOTVALID = 16,       /* = FINUFFT_ERR_PLAN_NOTVALID */
  SQN_ERR_NUM_NU_PTS_INVALID = 20,  /* = FINUFFT_ERR_NUM_NU_PTS_INVALID */
  SQN_ERR_INVALID_ARGUMENT = 21,    /* = FINUFFT_ERR_INVALID_ARGUMENT */
  SQN_ERR_ABI_MISMATCH = 40,        /* descriptor built against another ABI version */
  SQN_ERR_NO_DEVICE = 41,           /* no CUDA device, or device id out of range */
  SQN_ERR_GRID_TOO_LARGE = 42,      /* prod(modes) above max_grid_modes */
  SQN_ERR_NO_MODES = 43,            /* no reciprocal lattice point in [qmin, qmax] */
  SQN_ERR_DEGENERATE_CELL = 44,
  SQN_ERR_TYPE_ID = 45,             /* a type id outside 1..ntypes */
  SQN_ERR_CUFFT = 46,               /* cuFFT plan or execution failure */
  SQN_ERR_TIMEOUT = 47,             /* a bounded device wait gave up */
  SQN_ERR_NOT_SUPPORTED = 48,
  SQN_ERR_SCRATCH_LIMIT = 49,       /* request does not fit the fixed no-alloc scratch */
  SQN_ERR_DUMP = 50                 /* dump file unreadable or malformed (sqn_dump_last_error) */
};

enum { SQN_WEIGHT_UNIT = 0, SQN_WEIGHT_NEUTRON = 1, SQN_WEIGHT_XRAY = 2 };
/* Normalisations of src/sqc_structure_factor.f90:53-55. */
enum { SQN_NORM_MEAN = 1, SQN_NORM_SELF = 2, SQN_NORM_NATOM = 3 };
/* DOUBLE: FP64 spread / FFT / deconvolution.  SINGLE: FP32 spread / FFT /
 * deconvolution; pair products, |rho|^2, shell sums and normalisation FP64. */
enum { SQN_PREC_DOUBLE = 0, SQN_PREC_SINGLE = 1 };
/* Where a positions pointer lives. */
enum { SQN_HOST = 0, SQN_DEVICE = 1 };
/* sqn_plan_desc.flags */
enum {
  SQN_FLAG_TIMING = 1, /* record per-stage CUDA events (sqn_stage_times) */
  SQN_FLAG_GRAD = 2,   /* allocate the adjoint buffers of sqn_sq_grad */
  SQN_FLAG_CUFFT = 8,      /* cuFFT R2C + the bin kernel (instead of the pruned 512-point
                              passes that 512^3 grids use by default) */
  SQN_FLAG_AUTOTUNE = 128  /* choose the fine grid and kernel width by timing: the plan
                              builds the candidate (sigma, w) pairs that reach eps (the
                              smallest upsampling for each width up to the precision's
                              cap), runs a few frames of uniform synthetic positions of
                              its own shape through each, and keeps the fastest; results
                              are cached per shape for the life of the process.  Ignored
                              when upsampfac or kernel_width is given */
};

/* Everything sqcalc's configure + gpu_setup know after the first frame
 * (src/sqc_structure_factor.f90:313-422, src/sqc_gpu.f90:108-210). */
typedef struct sqn_plan_desc {
  int32_t abi_version;      /* SQN_ABI_VERSION */
  int32_t device;           /* CUDA device id (--gpu-id) */
  double cell[9];           /* lattice vectors, layout above (cell_t%a) */
  double origin[3];         /* cell_t%origin */
  int64_t natoms;
  const int32_t *type_id;   /* [natoms] LAMMPS type ids in 1..ntypes, host memory, copied */
  int32_t ntypes;           /* structure_factor_t%ntypes (largest type id) */
  int32_t weight;           /* SQN_WEIGHT_* (-w) */
  const double *amp_const;  /* [ntypes] neutron b per type id; NULL for unit / x-ray */
  const double *xray_coef;  /* [ntypes][9] IT92 a1..a4, b1..b4, c per type id; NULL unless x-ray */
  double qmin, qmax;        /* --qmin --qmax */
  int32_t nq;               /* --nq */
  int32_t norm;             /* SQN_NORM_* (--norm) */
  int32_t partials;         /* --partials (pair sums per type pair) */
  int32_t want_grid;        /* --grid (per-mode accumulators) */
  int32_t precision;        /* SQN_PREC_* (--precision) */
  int32_t flags;            /* SQN_FLAG_* */
  double eps;               /* NUFFT tolerance (--eps) */
  double upsampfac;         /* fine-grid upsampling sigma; 0 = chosen by the plan */
  int32_t kernel_width;     /* ES kernel width w; 0 = from eps and sigma */
  int32_t reserved;
  int64_t max_grid_modes;   /* prod(modes) cap; 0 = sqcalc's 4e8, < 0 = none */
  void *stream;             /* cudaStream_t to run on, or NULL for a plan-owned stream */
  /* Powder XRD pattern (--xrd, structure_factor_t%xrd_*,
   * src/sqc_structure_factor.f90:125-146): on when xrd_lambda > 0.  Bins uniform
   * in two-theta over [xrd_2theta_min, xrd_2theta_max] degrees, of width
   * xrd_step (<= 0: from the box, sf_configure_xrd :846-905, every direction
   * taken as periodic); each kept mode adds |total|^2 and the amplitude-weighted
   * pair products, times the Lorentz-polarization factor when xrd_lp. */
  double xrd_lambda;        /* incident wavelength, Angstrom (--xrd-lambda) */
  double xrd_2theta_min;    /* --xrd-range (default 1 .. 179) */
  double xrd_2theta_max;
  double xrd_step;          /* --xrd-step */
  int32_t xrd_lp;           /* --lp (1, default) / --no-lp (0) */
  int32_t reserved2;
} sqn_plan_desc;

/* What the plan chose. */
typedef struct sqn_plan_info {
  int32_t modes[3];         /* structure_factor_t%modes */
  int32_t kernel_width;
  int64_t nf[3];            /* fine grid */
  int64_t gridpoints;       /* prod(modes) */
  int64_t nmodes;           /* kept modes with qmin <= |q| <= qmax, q != 0 */
  double upsampfac;
  double beta;              /* ES shape parameter */
  double eps_used;
  int32_t ntransforms;      /* fine grids per frame: species count or 1 */
  int32_t nspecies;         /* type ids that have atoms */
  int64_t device_bytes;     /* device memory the plan holds */
  int64_t tile[3];          /* spread tile in fine-grid cells */
  int64_t natoms;           /* atoms per frame */
  int32_t xrd_bins;         /* two-theta bins of the powder pattern (0: off) */
  int32_t pruned_fft512;    /* 1: the frame FFT runs as pruned 512-point passes of ours
                               (every axis 512, no SQN_FLAG_CUFFT) instead of cuFFT */
  double xrd_step;          /* their width, degrees */
  int32_t autotuned;        /* 1: fine grid and width chosen by timing (SQN_FLAG_AUTOTUNE) */
  int32_t tune_candidates;  /* (sigma, w) pairs timed (0 when the choice came from the cache) */
  double tune_ms;           /* measured milliseconds per frame of the chosen pair */
} sqn_plan_info;

typedef struct sqn_plan_s sqn_plan;

/* ABI version of the loaded library (compare with SQN_ABI_VERSION). */
int sqn_abi_version(void);

/* Static text for a status code. */
const char *sqn_error_string(int code);

/* Descriptor defaults: sqcalc's option defaults (src/sqc_options.f90:51-140:
 * qmin 0, qmax 20, nq 500, eps 1e-9, norm mean, partials on, unit weights). */
void sqn_default_desc(sqn_plan_desc *desc);

/* Build the reciprocal grid, the shell map, den / shell_count and every device
 * buffer, and select the kernel.  Replaces sf_configure's grid setup plus
 * gpu_setup (src/sqc_gpu.f90:108-210: cudaMalloc of x, y, z, c, fk and
 * cufinufft[f]_makeplan).  *out is NULL on error. */
int sqn_plan_create(const sqn_plan_desc *desc, sqn_plan **out);

int sqn_plan_info_get(const sqn_plan *plan, sqn_plan_info *info);

/* Add nframes frames to the accumulators.  pos holds nframes consecutive
 * frame%pos(3, natoms) blocks in host (SQN_HOST) or device (SQN_DEVICE) memory.
 * Replaces one gpu_accumulate per frame (src/sqc_gpu.f90:213-362: host wrap,
 * uploads, cufinufft_setpts / execute, download, host pair sums and binning).
 * The call returns once the positions have been read; the transforms run
 * asynchronously on the plan's stream (device positions are read in the
 * plan's stream order and must stay valid until sqn_sync). */
int sqn_accumulate_frames(sqn_plan *plan, const double *pos, int64_t nframes, int32_t where);

/* Order everything queued so far before work the caller queues next on the
 * plan's stream (an event, a collective on the accumulators), without blocking
 * the host.  Every kernel of a plan runs on its one stream, so this only checks
 * the plan; it stays for callers written against a plan with several streams. */
int sqn_join(sqn_plan *plan);

/* Wait for all queued work of the plan. */
int sqn_sync(sqn_plan *plan);

/* Copy the accumulators out (syncs first).  Any pointer may be NULL.
 *   num[nq], den[nq], shell_count[nq]         structure_factor_t%num, den, shell_count
 *   partial_num[ntypes*ntypes*nq]             partial_num (zero when partials are off)
 *   gnum[gridpoints], gden[gridpoints]        gnum, gden (want_grid only)
 * Replaces reading the Fortran accumulators filled by sf_accumulate_values /
 * sf_accumulate_partials (src/sqc_structure_factor.f90:481-643). */
int sqn_get_accumulators(sqn_plan *plan, double *num, double *den, int64_t *shell_count,
                         double *partial_num, double *gnum, double *gden, int64_t *nframes);

/* Queue a device-to-host copy of num[nq] into host memory (pinned for an
 * asynchronous copy) after the queued frames, without waiting; it is complete
 * after sqn_sync. */
int sqn_peek_num_async(sqn_plan *plan, double *num_host);

/* Normalised results (syncs first); NULL pointers are skipped.
 *   S_total[nq]                         sf_shell_value  (:657-665)
 *   S_partial[ntypes*ntypes*nq]         sf_partial_value (:696-719), faber_ziman 0/1
 *   S_grid[nmodes]                      sf_grid_value (:757-768), kept modes in the
 *                                       reference's enumeration order (:352-381) */
int sqn_finalize(sqn_plan *plan, int32_t faber_ziman, double *S_total, double *S_partial,
                 double *S_grid, int64_t *nframes);

/* Zero the accumulators and the frame count. */
int sqn_reset(sqn_plan *plan);

/* The powder XRD pattern (plans with xrd_lambda > 0; syncs first), per atom
 * and per frame as sf_write_xrd writes it (src/sqc_structure_factor.f90:
 * 964-1031): two_theta[xrd_bins] bin centres (degrees), I[xrd_bins],
 * I_partial[ntypes*ntypes*xrd_bins] (first index fastest; a <= b filled, zero
 * without partials; I = sum_a I_aa + 2 sum_{a<b} I_ab), count[xrd_bins] kept
 * modes per bin (both mirrors counted; sf_xrd_empty_bins :927-936).  Any pointer
 * may be NULL. */
int sqn_get_xrd(sqn_plan *plan, double *two_theta, double *I, double *I_partial, int64_t *count,
                int64_t *nframes);

/* Density amplitudes of one frame at reciprocal lattice points, the per-frame
 * input of sqcalc dyn on a grid (--qpoints grid): rho_a(q_h) = sum_{j of type a}
 * exp(i q_h . r_j), which the reference sums directly, O(N nq) per frame
 * (dyn_accumulate, src/sqc_dynamics.f90:792-880); here all of them come from one
 * pass of the frame transforms.  hkl [nmodes][3] host int32 lattice indices with
 * |h_d| <= (modes_d - 1)/2 (others give 0); rho [nspecies][nmodes] host, as
 * interleaved (re, im) doubles, species in ascending type id.  Needs a plan with a
 * transform per species (partials or x-ray weights) on the cuFFT path; does not
 * touch the accumulators.  The plan's eps holds for |q_h| <= qmax; toward the corners
 * of the mode cube the deconvolution amplifies the grid's rounding (FP32 plans lose
 * digits there, FP64 plans stay near eps).  Synchronous. */
int sqn_density_modes(sqn_plan *plan, const double *pos, int32_t where, const int32_t *hkl,
                      int64_t nmodes, double *rho);

/* Frames sharded over ranks (one process per GPU, each with its own plan on
 * the same system).  The plan's FP64 sums -- shell sums, pair sums and, with
 * want_grid, the per-mode sums -- are one device buffer of *count doubles at
 * *acc (syncs first); *nframes receives the frames accumulated here.  The
 * caller adds the buffers of all ranks in place with one sum all-reduce
 * (ncclAllReduce on the device pointer), then calls sqn_set_frame_count with
 * the total so that sqn_finalize normalises over all frames.  Replaces nothing
 * in the reference, which reads one trajectory in one process
 * (src/sqc_structure_factor.f90:457-470 per frame). */
int sqn_accumulator_view(sqn_plan *plan, double **acc, int64_t *count, int64_t *nframes);
int sqn_set_frame_count(sqn_plan *plan, int64_t nframes);

/* Per-stage device time summed over the frames since the last reset, in ms:
 * out[0] wrap+bin sort, out[1] spread, out[2] FFT, out[3] deconvolve+bin,
 * out[4] frames timed.  Needs SQN_FLAG_TIMING. */
int sqn_stage_times(sqn_plan *plan, double *out, int32_t n);

/* One frame, outside the accumulators: S_frame(q) = sum_{h in shell} |T(h)|^2 / den
 * and, when dLdS is given, the gradient of L = sum_s dLdS[s] * S_frame(s) with
 * respect to the Cartesian positions (q-independent weights; the plan needs
 * SQN_FLAG_GRAD).  pos [natoms][3] and grad [natoms][3] live in host (SQN_HOST)
 * or device (SQN_DEVICE) memory; dLdS [nq] and S [nq] in host memory; S may be
 * NULL.  The forward transform is recomputed (nothing is kept from earlier
 * calls); the adjoint is three type-2 NUFFTs (amplify, C2R FFT, ES
 * interpolation).  No counterpart in the reference, which has no gradient;
 * it differentiates the direct sum of src/sqc_structure_factor.f90:1440-1456.
 * Synchronous. */
int sqn_sq_grad(sqn_plan *plan, const double *pos, int32_t where, const double *dLdS, double *S,
                double *grad);

/* Number of this library's own kernel launches so far (cuFFT's not counted). */
int64_t sqn_launch_count(const sqn_plan *plan);

/* ---- cuFINUFFT-shaped type-1 NUFFT ----------------------------------------
 * fk[t][k] = sum_j c[t][j] exp(iflag i (k1 x_j + k2 y_j + k3 z_j)) for
 * k_d in [-N_d/2, (N_d-1)/2], the type-1, dim-3 transform of
 * cufinufft[f]_makeplan / setpts / execute / destroy
 * (external/finufft/include/cufinufft.h, bound by sqcalc in
 * src/sqc_cufinufft.f90:183-259): the same arguments and life cycle, so the
 * library can stand in for those calls literally and be compared with them
 * transform for transform.  type must be 1 and dim 3 (else
 * SQN_ERR_NOT_SUPPORTED); n_modes[3] = (N1, N2, N3); iflag >= 0 means +1;
 * ntransf transforms share the points; tol as cuFINUFFT's tol.
 * setpts: M points, device arrays x, y, z (period 2 pi, any real value), sorted
 * once per call.  execute: device arrays c [ntransf][M] and fk
 * [ntransf][N3][N2][N1] of interleaved (re, im) doubles (floats for the f
 * variants), modes in opts.modeord order (0: -N/2 first, 1: 0 first).
 * execute is synchronous on the plan's stream. */
typedef struct sqn_type1_s sqn_type1_plan;
typedef struct sqn_type1_opts {
  int32_t gpu_device_id; /* cufinufft_opts.gpu_device_id */
  int32_t modeord;       /* cufinufft_opts.modeord: 0 CMCL order, 1 FFT order */
  double upsampfac;      /* 0: chosen by the plan; else > 1 */
  void *gpu_stream;      /* cufinufft_opts.gpu_stream; NULL: a plan-owned stream */
} sqn_type1_opts;
void sqn_type1_default_opts(sqn_type1_opts *opts);
int sqn_type1_makeplan(int32_t type, int32_t dim, const int64_t *n_modes, int32_t iflag,
                       int32_t ntransf, double tol, sqn_type1_plan **plan,
                       const sqn_type1_opts *opts);
int sqn_type1f_makeplan(int32_t type, int32_t dim, const int64_t *n_modes, int32_t iflag,
                        int32_t ntransf, float tol, sqn_type1_plan **plan,
                        const sqn_type1_opts *opts);
int sqn_type1_setpts(sqn_type1_plan *plan, int64_t M, const double *d_x, const double *d_y,
                     const double *d_z);
int sqn_type1f_setpts(sqn_type1_plan *plan, int64_t M, const float *d_x, const float *d_y,
                      const float *d_z);
int sqn_type1_execute(sqn_type1_plan *plan, const double *d_c, double *d_fk);
int sqn_type1f_execute(sqn_type1_plan *plan, const float *d_c, float *d_fk);
int sqn_type1_destroy(sqn_type1_plan *plan);

/* ---- LAMMPS dump ingest ----------------------------------------------------
 * A multithreaded reader of LAMMPS text dumps, the counterpart of
 * lammps_next_frame / resolve_columns (src/sqc_dump.f90:162-313, :502-552):
 * frames of ITEM: TIMESTEP / NUMBER OF ATOMS / BOX BOUNDS [xy xz yz] / ATOMS with
 * the columns id, type and x|xu, y|yu, z|zu in file order.  The file is
 * memory-mapped and each frame's atom lines are parsed by nthreads threads
 * (<= 0: all cores) with correctly rounded decimal conversion.
 * sqn_dump_next: fills natoms, timestep, bounds[9] (the three bound rows
 * lo hi [tilt]; may be NULL), pos [natoms][3], type_id [natoms] and ids [natoms]
 * (may be NULL) for at most capacity atoms; *natoms = 0 at the end of the file
 * (status SQN_OK); a frame larger than capacity returns SQN_ERR_INVALID_ARGUMENT
 * with *natoms set and the frame not consumed; a malformed frame returns
 * SQN_ERR_DUMP and sqn_dump_last_error gives the reference's ierr (4 structure or
 * TIMESTEP, 5 atom count, 6 box row, 7 ATOMS before its header, 8 atom line,
 * 9 missing column).
 * sqn_accumulate_dump: up to max_frames (< 0: all) frames of the dump into the
 * plan, parsing frame f + 1 on a host thread into a second pinned buffer while
 * the plan uploads and transforms frame f; every frame must have the plan's atom
 * count (else SQN_ERR_NUM_NU_PTS_INVALID; the plan's type ids stand, as the
 * reference's species set up once) and the box bounds ref_bounds[9] (NULL: those
 * of the first frame read) to 1e-6 relative (else SQN_ERR_DUMP with
 * sqn_dump_last_error 10, the reference driver's "box changes" stop); syncs
 * before returning.  The two pinned frame buffers belong to the dump handle:
 * allocated by the first call, reused by later ones, freed by sqn_dump_close. */
typedef struct sqn_dump_s sqn_dump;
int sqn_dump_open(const char *path, int32_t nthreads, sqn_dump **dump);
int sqn_dump_next(sqn_dump *dump, int64_t capacity, int64_t *natoms, int64_t *timestep,
                  double *bounds, double *pos, int32_t *type_id, int64_t *ids);
int sqn_dump_last_error(const sqn_dump *dump);
int sqn_dump_rewind(sqn_dump *dump);
int sqn_dump_close(sqn_dump *dump);
int sqn_accumulate_dump(sqn_plan *plan, sqn_dump *dump, int64_t max_frames,
                        const double *ref_bounds, int64_t *frames_done);

/* ---- Batches of independent systems ------------------------------------
 * Many uneven systems (each its own cell, atoms, types and grid) whose frames
 * are accumulated together: one plan per system, and one frame of EVERY system
 * captured once into a CUDA graph, so that a step over all systems is a single
 * graph launch.  When the systems share precision, transform count and weight
 * kind (and have no powder pattern), the graph runs each frame stage for all
 * systems in one launch: bin sort (three launches), spread (one launch over
 * every system's tiles and transforms), the systems' FFTs as parallel branches,
 * binning (one launch over every system's rows); otherwise the root stream
 * forks to one stream per system, each running its own frame path.  With
 * SQN_FLAG_AUTOTUNE in the descriptors each system's fine grid and width are
 * chosen by timing.  No counterpart in the reference, which runs one system
 * per process.
 *
 * sqn_batch_create: descs[nsystems] as for sqn_plan_create (same device; each
 *   desc's stream is ignored, its timing flag cleared); stream is the root
 *   stream (NULL: the batch creates one).
 * sqn_batch_accumulate: pos[k] holds nframes frames [nframes][natoms_k][3] of
 *   system k (host or device, all the same); per frame the positions are staged
 *   on the root stream and the graph is replayed.  Asynchronous for device
 *   positions.
 * sqn_batch_plan: the plan of system k (owned by the batch) for
 *   sqn_get_accumulators / sqn_finalize after sqn_batch_sync; do not accumulate
 *   on it directly while graph replays are in flight.
 * sqn_batch_graph_launches: graph replays so far.
 * sqn_batch_launch_count: kernels of this library launched by those replays
 *   (cuFFT's own kernels not counted).
 * sqn_batch_multi: 1 when the batch runs the multi-system launches, 0 when it
 *   runs one branch per system. */
typedef struct sqn_batch_s sqn_batch;
int sqn_batch_create(const sqn_plan_desc *descs, int32_t nsystems, void *stream,
                     sqn_batch **out);
int sqn_batch_accumulate(sqn_batch *batch, const double *const *pos, int64_t nframes,
                         int32_t where);
int sqn_batch_sync(sqn_batch *batch);
int sqn_batch_plan(sqn_batch *batch, int32_t system, sqn_plan **plan);
int64_t sqn_batch_graph_launches(const sqn_batch *batch);
int64_t sqn_batch_launch_count(const sqn_batch *batch);
int32_t sqn_batch_multi(const sqn_batch *batch);
int sqn_batch_destroy(sqn_batch *batch);

/* Size of the fixed device scratch array of sqn_spread_frame_noalloc (per GPU). */
#define SQN_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/* Wrap, bin-sort and spread one frame onto caller-provided fine grids WITHOUT
 * allocating any device memory.  No counterpart in the reference: it is for
 * callers that cannot call cudaMalloc -- a host framework that owns all device
 * memory through its own pool, a plugin inside an application that has already
 * reserved the device memory, a service that must keep a fixed footprint.
 *   pos       [natoms][3] FP64 Cartesian positions, device memory
 *   species   [natoms] grid index of each atom (0..ntr-1), host memory; every
 *             index is checked on the host before anything is queued
 *   ntr       1 .. 8 grids (more: SQN_ERR_INVALID_ARGUMENT)
 *   strength  [ntr] FP32 strength of the atoms of each grid, host memory
 *             (species and strength are copied with cudaMemcpyAsync on stream)
 *   cell, origin, nf[3], kernel_width, beta: as sqn_plan_info reports them
 *   grid      [ntr][nf3][nf2][nf1] FP32 output, device memory, x fastest;
 *             every cell is written (no zeroing needed)
 *   stream    cudaStream_t or NULL
 * Its scratch (bin counts and starts, per-atom keys, sorted point records)
 * lives in one file-scope device array of SQN_NOALLOC_SCRATCH_BYTES that every
 * GPU loading the library holds until exit; requests that do not fit return
 * SQN_ERR_SCRATCH_LIMIT.  The first call on a device resolves the array's
 * address with that device current; make it before any stream capture.  Calls
 * share the array (it keeps the last call's contents; counts are cleared each
 * call), so calls that overlap on the GPU race and must be serialised.
 * FP32 only; returns once the work is queued on `stream`. */
int sqn_spread_frame_noalloc(const double *pos, int64_t natoms, const uint8_t *species,
                             int32_t ntr, const float *strength, const double *cell,
                             const double *origin, const int64_t *nf, int32_t kernel_width,
                             double beta, float *grid, void *stream);

/* Release the plan and its device memory.  Replaces cufinufft_destroy plus the
 * cudaFree calls of gpu_finalize (src/sqc_gpu.f90:365-404). */
int sqn_plan_destroy(sqn_plan *plan);

#ifdef __cplusplus
}
#endif
#endif /* SQNUFFT_H */
