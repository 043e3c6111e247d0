/*
 * dsht.h -- C ABI of the B200-native DirectSHT forward transform (libdsht_b200.so).
 *
 * Computes a_lm = sum_i w_i conj(Y_lm(theta_i, phi_i)) for weighted points on the sphere
 * with the reference's spline scheme: FP64 Ylm/dYlm tables on Nx uniform nodes in
 * x = |cos theta| in [0, xmax], cubic Hermite interpolation, per-bin per-m sums, and a
 * per-m contraction; points with |cos theta| >= xmax are rotated by +90 deg about y,
 * transformed, and their alm rotated back.  Output alm are complex128 (interleaved
 * re, im) in Healpy order alm[m(2Nl-1-m)/2 + l], l < Nl, m <= l.
 *
 * Reference interfaces replaced (martinjameswhite/directsht):
 *   dsht_plan_create      DirectSHT.__init__            sht/sht.py:32-56
 *   dsht_execute          DirectSHT.__call__ / basic_sht sht/sht.py:112-150, :153-283
 *   dsht_execute_maps     __call__ / basic_sht looped over weight maps of one point set
 *   dsht_execute_batch    __call__ / basic_sht looped over point sets of one (Nl, Nx)
 *   dsht_get_row          DirectSHT.get_Ylm / get_dYlm  sht/sht.py:69-93
 *   dsht_alm2cl           DirectSHT.alm2cl              sht/sht.py:95-109
 *   dsht_index            DirectSHT.indx                sht/sht.py:58-67
 *   dsht_mode_coupling    MaskDeconvolution.get_M       sht/mask_deconvolution.py:171-192
 *   dsht_make_table       make_table   (ctypes)         csht/sht_helper.c:18, csht/sht.py:39-42
 *   dsht_do_transform     do_transform (ctypes)         csht/sht_helper.c:176, csht/sht.py:111-115
 *
 * All functions return DSHT_OK (0) or a DSHT_ERR_* code; dsht_last_error() gives the
 * message of the last failure on the calling thread.  Device pointers are owned by the
 * caller; a plan owns its tables.  A plan may be shared read-only by several threads;
 * calls on one plan with the plan-owned workspace must not overlap.
 */
#ifndef DSHT_H_
#define DSHT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsht_plan_s* dsht_plan_t;

enum {
  DSHT_OK = 0,
  DSHT_ERR_INVALID = 1,      /* bad argument (sizes, null pointers)                  */
  DSHT_ERR_CUDA = 2,         /* CUDA runtime failure                                  */
  DSHT_ERR_NOMEM = 3,        /* device allocation or workspace too small              */
  DSHT_ERR_THETA_RANGE = 4,  /* basic_sht assertion: theta outside (acos xmax, acos -xmax)
                                (sht/sht.py:171-172) -> AssertionError                 */
  DSHT_ERR_EMPTY = 5,        /* basic_sht with no points (sht/sht.py:205-206) -> ValueError */
  DSHT_ERR_POLAR_RANGE = 6   /* a rotated polar point is still polar (xmax < sin(pi/4));
                                the reference then returns zeros (sht/sht.py:141-148)   */
};

/* Execution modes of dsht_execute. */
enum {
  DSHT_MODE_CALL = 0,   /* DirectSHT.__call__: polar/equatorial split + rotation   */
  DSHT_MODE_BASIC = 1   /* DirectSHT.basic_sht: every point must be equatorial     */
};

/* Plan flags.  DSHT_PLAN_F32_TABLES: keep only the compact 4-byte fixed-point tables (each
 * row of Yv and dx*Yd as 31-bit integers of one power-of-two row scale, stored as four int8
 * digit planes; built from the FP64 recurrences a few columns at a time; half the memory of
 * the FP64 pair: 68.7 GB instead of 137 GB at Nl=2048, Nx=4096).  Such a plan runs at
 * DSHT_PREC_MIXED only (transforms below DSHT_MIXED_MIN_POINTS points use FP64 bin sums with
 * the compact tables); dsht_get_row / dsht_get_table return the stored values, within
 * 2^-31 of their row's largest entry.  Needs Nx <= 8192 and Nl <= 2048. */
enum {
  DSHT_PLAN_DEFAULT = 0,
  DSHT_PLAN_F32_TABLES = 1
};

/* Arithmetic of a plan's transforms.
 *   DSHT_PREC_FP64  : FP64 CUDA-core per-bin sums and FP64 tables; agrees with the
 *                     reference's numpy path to about 1e-15 (tested at <= 1e-12 x max|alm|).
 *   DSHT_PREC_MIXED : per-bin sums (see DSHT_TUNE_BIN_SUMS for the choice) by a type-1
 *                     non-uniform FFT in FP64 (each bin's points
 *                     spread onto a periodic grid of 4 x 2^ceil(log2 Nl) cells with a width-12
 *                     "exponential of semicircle" kernel, FFT, division by the kernel's Fourier
 *                     transform; error about 5e-12 of the bin's sum of |w h_k|) -- or the
 *                     direct tcgen05 tensor-core
 *                     sums (operands quantised to 22-bit fixed point, split into int8 slices,
 *                     slice products accumulated exactly in S32 and combined in FP64;
 *                     unbiased, about 5.6e-8 rms per product) -- and a
 *                     tcgen05 tensor-core contraction of 4-byte fixed-point copies of the
 *                     tables (31-bit digits per row and per fold column, five exact S32
 *                     digit-pair classes; contraction error about 1e-9 x max|alm|), built on
 *                     first use; every table tile is read once for up to eight maps or point
 *                     sets of a multi-transform call.  Within 1e-7 x max|alm| of FP64,
 *                     concentrated point sets included.  With the tensor-core sums the
 *                     fixed-point scale of a bin piece is its largest |weight|: weights
 *                     spanning many decades lose accuracy (lognormal sigma <= 1.5 stays within
 *                     1e-7), and so do weights of both signs whose sums cancel (zero-mean
 *                     normal weights: ~3e-7); the NUFFT sums have neither limit.
 *                     Plans with Nx > 8192 (or without room for the digit tables beside the
 *                     FP64 pair) contract the FP64 tables instead.
 *   DSHT_PREC_MIXED_F64_TABLES : the same bin sums with the FP64 tables streamed by the
 *                     CUDA-core contraction.
 * Mixed levels need Nl <= 2048; transforms of fewer than DSHT_MIXED_MIN_POINTS points run
 * the FP64 stages (they cost little, and the quantisation error of a handful of points
 * does not average down).  The rotation stays FP64 in all levels. */
enum {
  DSHT_PREC_FP64 = 0,
  DSHT_PREC_MIXED = 1,
  DSHT_PREC_MIXED_F64_TABLES = 2
};
#define DSHT_MIXED_MIN_POINTS 1024
int64_t dsht_mixed_min_points(void);
int dsht_set_precision(dsht_plan_t plan, int precision);
int dsht_get_precision(dsht_plan_t plan, int* precision);

/* Tuning of a plan (no counterpart in the reference; results do not depend on it beyond
 * the stated precision).  DSHT_TUNE_PIECE_MAX: points per bin piece of the per-bin sums, a
 * multiple of 32 in [256, 65536], 0 = chosen from N and the method (the direct sums, FP64 and
 * tensor-core, cap it at 2048; the NUFFT sums default to 8192).  DSHT_TUNE_MAPS_PER_PASS:
 * maps or point sets that share one read of the tables in a multi-transform call, 1..8,
 * 0 = the most (8; the tensor-core contraction only: the FP64 one reads the tables once per
 * map).  DSHT_TUNE_BIN_SUMS: the bin sums of the mixed levels, DSHT_BIN_SUMS_NUFFT,
 * DSHT_BIN_SUMS_TC (the direct int8-slice tensor-core sums) or DSHT_BIN_SUMS_FP64 (the direct
 * FP64 CUDA-core sums of the fp64 level); AUTO (the default) chooses per transform (so the
 * transforms of one batch call may differ) from its points per bin key on average: the
 * NUFFT sums from 512 (N >= 2048 (Nx - 1)), where their fixed cost per bin piece pays off,
 * the FP64 direct sums below 28 (N < 112 (Nx - 1): pieces of a few points, where the
 * tensor-core sums' per-piece GEMM tile costs more than FP64 work per point), and the
 * tensor-core sums in between.  Workspace sizes depend on all three: query them after
 * tuning. */
enum { DSHT_TUNE_PIECE_MAX = 1, DSHT_TUNE_MAPS_PER_PASS = 2, DSHT_TUNE_BIN_SUMS = 3 };
/* Values of DSHT_TUNE_BIN_SUMS: the bin-sum method of the mixed levels. */
enum { DSHT_BIN_SUMS_AUTO = 0, DSHT_BIN_SUMS_NUFFT = 1, DSHT_BIN_SUMS_TC = 2, DSHT_BIN_SUMS_FP64 = 3 };
int dsht_plan_tune(dsht_plan_t plan, int param, int value);
int dsht_plan_get_tune(dsht_plan_t plan, int param, int* value);

/* Build the x grid and the FP64 Ylm/dYlm tables on the current CUDA device.
 * Replaces DirectSHT.__init__ (sht/sht.py:32-56). 1 <= Nl <= 16384, 2 <= Nx <= 12288 (the sort histograms
 * 4 (Nx - 1) bin keys in shared memory), 0 < xmax < 1. */
int dsht_plan_create(int Nl, int Nx, double xmax, int flags, dsht_plan_t* plan);
int dsht_plan_destroy(dsht_plan_t plan);

/* Sizes of a plan. */
int dsht_plan_info(dsht_plan_t plan, int* Nl, int* Nx, double* xmax, int64_t* Nlm);

/* Healpy index m(2Nl-1-m)/2 + l (sht/sht.py:58-67). */
int64_t dsht_index(int Nl, int ell, int m);

/* Bytes of device workspace dsht_execute needs for N points. */
int dsht_workspace_size(dsht_plan_t plan, int64_t N, size_t* bytes);

/* Forward transform of N points given by DEVICE pointers theta, phi, w (float64).
 * alm: DEVICE pointer to 2*Nlm doubles (complex128), overwritten.
 * workspace: DEVICE buffer of at least dsht_workspace_size bytes, or NULL to use a
 * buffer the plan owns (grown on demand).  stream: a cudaStream_t (NULL = default).
 * Stream-ordered; range errors are detected on the device and reported when the call
 * synchronises, which it does once at the end (to read the error flags).
 * Replaces DirectSHT.__call__ (mode CALL) and DirectSHT.basic_sht (mode BASIC). */
int dsht_execute(dsht_plan_t plan, const double* theta, const double* phi, const double* w,
                 int64_t N, int mode, double* alm, void* workspace, size_t workspace_bytes,
                 void* stream);

/* Weight dtypes of dsht_execute_maps. */
enum { DSHT_W_F64 = 0, DSHT_W_F32 = 1 };

/* Bytes of device workspace dsht_execute_maps needs for N points and nmaps maps. */
int dsht_workspace_size_maps(dsht_plan_t plan, int64_t N, int nmaps, size_t* bytes);

/* nmaps weight maps on one point set: alm of map k = DirectSHT(theta, phi, w_k)
 * with w_k = the N weights at w + k * w_stride ELEMENTS, float64 or float32 (w_dtype);
 * float32 weights are widened to float64 exactly.  theta, phi, w: DEVICE pointers.
 * alm: DEVICE pointer to nmaps * 2 * Nlm doubles, map k at alm + k * 2 * Nlm.  The
 * reference has no multi-map call: a user loops DirectSHT.__call__ (sht/sht.py:112-150)
 * or basic_sht over the maps with the same theta, phi, and gets the same alm.  Here the
 * points are classified and sorted once.  Other arguments as dsht_execute. */
int dsht_execute_maps(dsht_plan_t plan, const double* theta, const double* phi, const void* w,
                      int w_dtype, int64_t N, int nmaps, int64_t w_stride, int mode, double* alm,
                      void* workspace, size_t workspace_bytes, void* stream);

/* dsht_execute_maps without synchronisation, for CUDA-graph capture and overlapped
 * streams: needs a caller workspace, allocates nothing, waits for nothing.  The device
 * word *status (may be NULL) receives the transform's flags when the work has run;
 * dsht_status(flags, mode) turns them into the DSHT_* code dsht_execute_maps would return. */
int dsht_enqueue_maps(dsht_plan_t plan, const double* theta, const double* phi, const void* w,
                      int w_dtype, int64_t N, int nmaps, int64_t w_stride, int mode, double* alm,
                      unsigned* status, void* workspace, size_t workspace_bytes, void* stream);
int dsht_status(unsigned flags, int mode);

/* Batches of independent transforms on one plan (no counterpart in the reference, whose
 * users call DirectSHT.__call__ once per point set).  Transform i: N[i] points at the
 * DEVICE pointers theta[i], phi[i], w[i] (float64), alm to the DEVICE pointer alm[i]
 * (2*Nlm doubles); the pointer arrays themselves are HOST arrays read during the call.
 * Each point set is sorted on its own; the contraction serves up to 8 transforms per read
 * of the digit tables (DSHT_TUNE_MAPS_PER_PASS; one per read of FP64 tables) and the
 * rotation up to 8.  Results equal those of one dsht_execute per transform.  The workspace (dsht_workspace_size_batch with the
 * largest N of the batch) is used in turn by every transform.  dsht_execute_batch
 * synchronises and returns the first error of any transform; dsht_enqueue_batch does not
 * synchronise, allocates nothing, and writes the flags of transform i to the DEVICE word
 * status[i] (status may be NULL). */
int dsht_workspace_size_batch(dsht_plan_t plan, int64_t max_N, int ntrans, size_t* bytes);
int dsht_execute_batch(dsht_plan_t plan, int ntrans, const double* const* theta,
                       const double* const* phi, const double* const* w, const int64_t* N,
                       int mode, double* const* alm, void* workspace, size_t workspace_bytes,
                       void* stream);
int dsht_enqueue_batch(dsht_plan_t plan, int ntrans, const double* const* theta,
                       const double* const* phi, const double* const* w, const int64_t* N,
                       int mode, double* const* alm, unsigned* status, void* workspace,
                       size_t workspace_bytes, void* stream);

/* alm_out = alm_add + R(alm_rot): alm of points rotated by +90 deg about y rotated back to
 * the original frame with Wigner d(pi/2) (DEVICE pointers, 2*Nlm doubles each; alm_add may be
 * NULL for zeros, alm_out may alias alm_add).  Replaces healpy's
 * Rotator(rot=(0,90,0), eulertype='ZYZ', inv=True).rotate_alm at sht/sht.py:138-139. */
int dsht_rotate_back(dsht_plan_t plan, const double* alm_rot, const double* alm_add, double* alm_out,
                     void* stream);

/* dsht_execute without any allocation.  No counterpart in the reference.  For callers that
 * cannot allocate device memory when they run a transform: a framework that has reserved
 * nearly all GPU memory for its own pool, a plugin host that forbids plugins to allocate,
 * or a latency-critical loop that cannot afford the device-wide synchronisation of
 * cudaMalloc/cudaFree.  Same arguments and results as dsht_execute (DEVICE pointers), but
 * all scratch lives in one fixed device array of dsht_noalloc_scratch_bytes() = 64 MiB
 * that every GPU loading this library holds until exit; problems whose workspace is larger
 * return DSHT_ERR_NOMEM.  With the default piece size, Nl=256, Nx=512, N=1e5 fits (63.8 MB);
 * a plan tuned to smaller pieces (DSHT_TUNE_PIECE_MAX) needs more: check a problem with
 * dsht_workspace_size(plan, N) <= dsht_noalloc_scratch_bytes() beforehand.  Like
 * dsht_execute, each call waits for its stream once at the end to read the error flags,
 * and N is limited to 0xfffffff0 points; because of that wait a call can never be captured
 * into a CUDA graph (dsht_enqueue_maps is the capturable entry point).  All
 * calls share the array (it keeps the last call's contents; what must start at zero is
 * cleared), so calls that overlap on the GPU race and must be serialised by the caller. */
int dsht_execute_noalloc(dsht_plan_t plan, const double* theta, const double* phi, const double* w,
                         int64_t N, int mode, double* alm, void* stream);
size_t dsht_noalloc_scratch_bytes(void);

/* Same with HOST pointers (pageable or pinned); copies in, runs, copies alm out. */
int dsht_execute_host(dsht_plan_t plan, const double* theta, const double* phi,
                      const double* w, int64_t N, int mode, double* alm_host);

/* One row of the tables to HOST memory: which = 0 -> Ylm(x_j, 0), 1 -> dYlm/dx.
 * out: Nx doubles.  Replaces DirectSHT.get_Ylm / get_dYlm (sht/sht.py:69-93). */
int dsht_get_row(dsht_plan_t plan, int which, int ell, int m, double* out);

/* Whole table (Nlm x Nx doubles) to a HOST buffer. */
int dsht_get_table(dsht_plan_t plan, int which, double* out);

/* Whole table in the JAX path's layout, out[m][l - m][j] (Nl x Nl x Nx doubles), with the
 * entries l >= Nl set to zero (null_unphysical).  Replaces the (Nell, Nell, Nx) Yv/Yd
 * attributes of DirectSHT when JAX is present (sht/sht.py:49-55, sht/legendre_jax.py:14-25;
 * get_Ylm reads Yv[m, ell-m, :] there, sht/sht.py:77-80).  out_on_device = 0: out is a HOST
 * buffer (synchronous); 1: a DEVICE buffer, filled by a kernel on `stream`. */
int dsht_get_table_mlayout(dsht_plan_t plan, int which, double* out, int out_on_device, void* stream);

/* Pseudo-spectrum cl[l] = (|a_l0|^2 + 2 sum_{m>0} |a_lm|^2)/(2l+1) of a HOST alm vector.
 * Replaces DirectSHT.alm2cl (sht/sht.py:95-109). */
int dsht_alm2cl(int Nl, const double* alm, double* cl);

/* The same pseudo-spectrum for nmaps alm vectors already on the device, without copying
 * them to the host.  alm: DEVICE pointer, map k at alm + k * alm_stride doubles (each 2*Nlm
 * doubles, complex128 Healpy order); cl: DEVICE pointer to nmaps * Nl doubles, map k's
 * spectrum at cl + k * Nl.  Stream-ordered on `stream` (NULL = default), no synchronisation.
 * Replaces DirectSHT.alm2cl (sht/sht.py:95-109) for device-resident alm. */
int dsht_alm2cl_device(int Nl, int nmaps, const double* alm, int64_t alm_stride, double* cl, void* stream);

/* Mode-coupling matrix of pseudo-Cl for a window W: M[l1 * Nl + l2] =
 * (2 l2 + 1)/(4 pi) sum_{l3} (2 l3 + 1) W[l3] (l1 l2 l3; 0 0 0)^2 for l1, l2 < Nl, with
 * W[l3] = 0 for l3 >= nW.  W: DEVICE pointer to nW doubles; M: DEVICE pointer to Nl*Nl
 * doubles.  Stream-ordered on `stream`, no synchronisation.  Replaces
 * MaskDeconvolution.get_M (sht/mask_deconvolution.py:171-192) and the Wigner 3j table it
 * reads (sht/threej000.py:9-41, 76-117): the symbols are formed on the fly. */
int dsht_mode_coupling(int Nl, const double* W, int nW, double* M, void* stream);

/* Drop-ins for the reference's ctypes library csht/sht_helper.so (HOST arrays).
 * dsht_make_table fills Yv, Yd (Nlm*Nx doubles each) like make_table
 * (csht/sht_helper.c:18-116).  dsht_do_transform takes points of one sign of cos(theta)
 * (cost = cos(theta)), accumulates nothing across calls, and writes
 * carr = sum w Y cos(m phi), sarr = sum w Y sin(m phi) per Healpy index with
 * |cos theta| interpolated and no parity factor, like do_transform
 * (csht/sht_helper.c:176-286); Yv/Yd are not read: the tables of a plan cached per
 * (Nl, Nx, xmax) on the device are used.  Return 0 on success, like the reference. */
int dsht_make_table(int Nl, int Nx, double xmax, double* Yv, double* Yd);
int dsht_do_transform(int Nl, int Nx, double xmax, double* Yv, double* Yd, int Np,
                      double* cost, double* phi, double* wt, double* carr, double* sarr);

/* Stage timers (CUDA events recorded on the execute stream at every stage boundary).
 * Stages: 0 points+sort, 1 bin sums, 2 fold, 3 contraction, 4 rotation.  Each stage's time
 * is the sum over all its launches in the call: for multi-map and batch calls stage 0 is
 * every sort, stage 1 every bin-sum launch (with the weight gathers of later maps), stage 2
 * every fold, stage 3 every contraction pass and stage 4 every rotation.  The synchronising
 * entry points (dsht_execute*) add their stages when they return; the stages of the last
 * dsht_enqueue_* call are added by the next dsht_profile_read once the caller has
 * synchronised that call's stream.  Calls on one plan must not overlap while profiling. */
enum { DSHT_STAGE_POINTS = 0, DSHT_STAGE_BIN_SUMS = 1, DSHT_STAGE_FOLD = 2, DSHT_STAGE_CONTRACT = 3,
       DSHT_STAGE_ROTATE = 4, DSHT_STAGE_COUNT = 5 };
int dsht_profile_enable(dsht_plan_t plan, int enable);
/* Accumulated milliseconds per stage and number of profiled executes; reset=1 clears. */
int dsht_profile_read(dsht_plan_t plan, double* ms, int64_t* calls, int reset);

/* Test hook, no counterpart in the reference: the next tensor-core contraction launch (any
 * plan, any thread) withholds one of its internal signals, so a bounded wait inside it runs
 * out after about one second; the kernel then stops cleanly, the device stays usable, and the
 * call returns DSHT_ERR_CUDA ("timed out").  Lets a test check that a stalled tensor-core
 * pipeline is reported instead of hanging. */
int dsht_test_stall_next_contraction(void);

/* Test hook, no counterpart in the reference: the sort key of every point as the transform
 * computes it (DEVICE pointers; keys[N] uint32, flags one unsigned), so tests can check the
 * binning index for index.  key = set * (Nx - 1) + bin with set 0/1 for equatorial points
 * of cos(theta) >= 0 / < 0 and 2/3 for rotated polar points of rotated x >= 0 / < 0, bin =
 * numpy.digitize(|x|, x_grid) - 1 (sht/sht.py:212); 0xffffffff for a point in no set.
 * flags holds the DSHT flag bits the call would raise. */
int dsht_test_point_keys(dsht_plan_t plan, const double* theta, const double* phi, int64_t N, int mode,
                         uint32_t* keys, unsigned* flags, void* stream);

/* Test hook, no counterpart in the reference: the host-side tables of the NUFFT bin sums for
 * Nl <= 2048 -- *logn = log2 of the grid cells, poly[12][12] the monomial coefficients (in
 * s = 2f - 1) of the kernel values at the 12 cells next to a point of fractional cell offset
 * f, dinv[Nl] = 1 / Psi(m).  Needs no GPU. */
int dsht_test_nufft_tables(int Nl, int* logn, double* poly, double* dinv);

/* Kernels this library has launched in this process (all devices). */
int64_t dsht_launch_count(void);

/* Message of the last error on this thread ("" if none). */
const char* dsht_last_error(void);

/* Library version string. */
const char* dsht_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DSHT_H_ */
