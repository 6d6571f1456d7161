/*
 * hydro_b200.h -- C ABI of libhydro_b200.so, the B200 (sm_100a) implementation
 * of HydroC's dimensionally split Godunov/MUSCL time step.
 *
 * Two groups of entry points:
 *
 * 1. The reference's own hot-path entry points, with the exact signatures of
 *    HydroC/HydroC99_2Domp/Src (real_t = double).  A program built against the
 *    reference links this library in place of hydro_godunov.c and the files
 *    the reference Makefile lists as offloadable (SRC2, Makefile:118-119).
 *    The state Hv->uold stays host memory owned by the caller; the library
 *    keeps a device-resident mirror keyed by that pointer (uploaded on first
 *    use, copied back by hydro_b200_sync_to_host or, with the environment
 *    variable HYDRO_B200_SYNC=1, after every hydro_godunov call).
 *    Hw / Hvw (the reference's host work arrays) are accepted and ignored.
 *
 * 2. hydro_b200_* extensions: explicit residency control, a device-resident
 *    multi-step driver, error reporting and a device-pointer level API.
 *
 * The reference functions return void and abort on failure.  Here they record
 * a thread-local error (hydro_b200_last_error) and return; with
 * HYDRO_B200_STRICT=1 in the environment they print the error and abort().
 * All entry points are meant to be called from one host thread.
 */
#ifndef HYDRO_B200_H
#define HYDRO_B200_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Types.  When the reference's parametres.h was included first (its guard
 * PARAMETRES_H_INCLUDED is defined) its definitions are used; otherwise these
 * layout-identical ones are (parametres.h:31-122; the layout is checked field
 * by field against the reference in tests/test_abi.py).
 * ------------------------------------------------------------------------ */
#ifndef PARAMETRES_H_INCLUDED
typedef double real_t;

enum { HB_XMIN_BOX, HB_XMAX_BOX, HB_YMIN_BOX, HB_YMAX_BOX, HB_UP_BOX, HB_DOWN_BOX,
       HB_LEFT_BOX, HB_RIGHT_BOX, HB_MAX_BOX };

typedef struct _hydroparam {
    int prt;
    real_t t, tend;
    int nstep, nstepmax;
    int noutput;
    real_t dtoutput;
    int nimage;
    real_t dtimage;
    int imin, imax, jmin, jmax, nx, ny, nxt, nyt, nxyt, nxystep;
    int nproc, mype;
    int globnx, globny;
    int box[HB_MAX_BOX];
    int nvar;
    real_t dx;
    real_t gamma;
    real_t courant_factor;
    real_t smallc, smallr;
    int niter_riemann;
    int iorder;
    real_t slope_type;
    int scheme;
    int boundary_right, boundary_left, boundary_down, boundary_up;
    int testCase;
    int shrinkSize;
    int shrink;
    FILE *fp;
} hydroparam_t;

#define HSCHEME_MUSCL 1
#define HSCHEME_PLMDE 2
#define HSCHEME_COLLELA 3

typedef struct _hydrovar {
    real_t *uold; /* [nvar][nyt][nxt], index i + nxt*(j + nyt*v) */
} hydrovar_t;

typedef struct _hydrovarwork {
    real_t *u, *q, *qxm, *qxp, *dq;
    real_t *qleft, *qright, *qgdnv, *flux;
} hydrovarwork_t;

typedef struct _hydrowork {
    real_t *c;
    real_t *e;
    real_t *tmpm1, *tmpm2;
    real_t *rl, *ul, *pl, *cl, *wl;
    real_t *rr, *ur, *pr, *cr, *wr;
    real_t *ro, *uo, *po, *co, *wo;
    real_t *rstar, *ustar, *pstar, *cstar;
    real_t *spin, *spout, *ushock;
    int *sgnm;
    int *goon;
    real_t *frac, *scr, *delp, *pold;
    int *ind, *ind2;
} hydrowork_t;
#endif /* PARAMETRES_H_INCLUDED */

/* ------------------------------------------------------------------------
 * 1. Reference entry points (drop-in).
 * ------------------------------------------------------------------------ */

/* Replaces hydro_godunov.c:26-145 (declared hydro_godunov.h:4-5): two sweeps,
 * x then y for idim == 1, y then x for idim == 2, each one fused kernel
 * (ghost fill, gather, constoprim, equation_of_state, slope, trace,
 * qleftright, riemann, cmpflx, update).  With idim == 2 the Courant maxima of
 * the resulting state are reduced inside the second sweep and cached for the
 * next compute_deltat. */
void hydro_godunov(int idim, real_t dt, const hydroparam_t H, hydrovar_t *Hv, hydrowork_t *Hw,
                   hydrovarwork_t *Hvw);

/* Replaces compute_deltat.c:31-77 (declared compute_deltat.h:10-11):
 * *dt = courant_factor*dx / max(max|c+u|, max|c+v|, smallc) over the interior. */
void compute_deltat(real_t *dt, const hydroparam_t H, hydrowork_t *Hw, hydrovar_t *Hv,
                    hydrovarwork_t *Hvw);

/* Replaces make_boundary.c:21-206 (declared make_boundary.h:6): fills the two
 * ghost layers of direction idim on the device mirror. */
void make_boundary(int idim, const hydroparam_t H, hydrovar_t *Hv);

/* Replaces vtkfile.c:140-352 (declared vtkfile.h:3): the same files
 * (Dep/XXXX/YY/Hydro_<pe>_<step>.vtr, the .pvtr header on rank 0, Hydro.pvd),
 * byte for byte, written from the device mirror of Hv->uold: the float
 * conversion and base64 encoding run on the GPU, so no host copy of the state
 * is needed.  Link it by leaving vtkfile.c out of the reference's objects.
 * Unlike the reference it creates the directories on every rank and has no
 * MPI barriers. */
void vtkfile(int step, const hydroparam_t H, hydrovar_t *Hv);

/* Replace compute_deltat.c:15-29 (declared compute_deltat.h:7-8).  init_mem
 * allocates nothing (the device path needs no host work arrays) and sets the
 * pointers to NULL; clean_mem copies every device mirror back to its host
 * array and releases it (the reference driver calls it once, after the time
 * loop: main.c:500). */
void compute_deltat_init_mem(const hydroparam_t H, hydrowork_t *Hw, hydrovarwork_t *Hvw);
void compute_deltat_clean_mem(const hydroparam_t H, hydrowork_t *Hw, hydrovarwork_t *Hvw);

/* ------------------------------------------------------------------------
 * 2. Extensions.
 * ------------------------------------------------------------------------ */

/* Error codes. */
#define HB_OK 0
#define HB_ERR_ARG 1        /* invalid argument / unsupported parameter set */
#define HB_ERR_CUDA 2       /* a CUDA runtime call failed */
#define HB_ERR_NODEV 3      /* no CUDA device */
#define HB_ERR_NOMEM 4      /* device allocation failed */
#define HB_ERR_STATE 5      /* non-finite or non-positive density detected */
#define HB_ERR_TIMEOUT 6    /* a bounded device-side wait gave up */

int hydro_b200_last_error(void);
const char *hydro_b200_last_error_message(void);
void hydro_b200_clear_error(void);

/* Residency of the mirror keyed by Hv->uold. */
int hydro_b200_sync_to_host(const hydroparam_t *H, hydrovar_t *Hv);   /* device -> host */
int hydro_b200_sync_to_device(const hydroparam_t *H, hydrovar_t *Hv); /* host -> device */
int hydro_b200_release(hydrovar_t *Hv); /* frees the mirror (no copy back) */
/* Stream (a cudaStream_t) on which the mirror of Hv->uold runs; creates and
 * uploads the mirror if needed. */
void *hydro_b200_mirror_stream(const hydroparam_t *H, hydrovar_t *Hv);

/* Device-resident driver loop with the semantics of main.c:344-408: from
 * (*t, *nstep, *dt) run until t >= tend or nstep >= nstepmax, recomputing dt
 * on even steps (halved at step 0), x->y sweeps on even steps and y->x on odd
 * steps, with dt and t kept on the device (no host synchronisation inside
 * the loop).  dts (optional, nstepmax - *nstep entries) receives the dt of each
 * step.  Returns the number of steps done, or -1 on error. */
int hydro_b200_run(const hydroparam_t *H, hydrovar_t *Hv, int nstepmax, real_t tend, real_t *t,
                   int *nstep, real_t *dt, real_t *dts);

/* Device-pointer level API (no host state involved).  A "domain" owns a
 * device state in the reference layout plus its scratch buffer, stream and
 * device clock.  The stream is returned as a void* (a cudaStream_t). */
typedef struct hb_domain hb_domain;
hb_domain *hydro_b200_domain_create(const hydroparam_t *H);
void hydro_b200_domain_destroy(hb_domain *d);
double *hydro_b200_domain_state(hb_domain *d); /* device pointer, 4*nxt*nyt doubles */
void *hydro_b200_domain_stream(hb_domain *d);
int hydro_b200_domain_upload(hb_domain *d, const double *host);    /* async on the stream */
int hydro_b200_domain_download(hb_domain *d, double *host);        /* async on the stream */
int hydro_b200_domain_synchronize(hb_domain *d);
int hydro_b200_domain_godunov(hb_domain *d, int idim, double dt, int fuse_courant);
int hydro_b200_domain_make_boundary(hb_domain *d, int idim);
int hydro_b200_domain_courant(hb_domain *d, double *cournox, double *cournoy); /* synchronous */

/* Domain split (the reference's MPI build of the same variant: SplitSurface.c,
 * mpibounds.c:165-310 called from make_boundary.c:48-52 and :125-129, the dt
 * MPI_Allreduce of main.c:361-372).  A subdomain's sides that face a neighbour
 * carry boundary type 0 (parametres.c:318-330): their ghost cells are not
 * filled by make_boundary but received from the neighbour before each sweep.
 *
 * hydro_b200_domain_sweep runs ONE sweep of a step: stage 0 is the step's
 * first sweep (direction idim), stage 1 its second.  A step is
 * sweep(0, first) then sweep(1, second), the same work as
 * hydro_b200_domain_godunov; fuse_courant (stage 1 only) reduces the Courant
 * maxima of the result for the next hydro_b200_domain_courant.
 *
 * Halo strips: hydro_b200_domain_halo_count(d, idim) doubles, the two
 * interior lines next to side (0 = left/down, 1 = right/up) of direction idim
 * over the interior lines of the other direction.  pack reads the state the
 * given stage's sweep reads (stage 0: the step's input; stage 1: the first
 * sweep's output); unpack writes the ghost cells of that side.  A neighbour's
 * strip of side 1-s unpacked at side s places its cells exactly where a single
 * grid holds them.  Buffers are device pointers; all three run asynchronously
 * on the domain's stream. */
int hydro_b200_domain_sweep(hb_domain *d, int stage, int idim, double dt, int fuse_courant);
/* The same sweep in two parts, so that a split can overlap its halo exchange
 * with the sweep: part 1 sweeps the windows of every line that read no ghost
 * cell (it may run before the halos of that sweep are unpacked), part 2 the
 * windows that do (after the unpack); part 0 is the whole sweep.  Parts 1
 * then 2 do the work of one hydro_b200_domain_sweep, with the same results.
 * With fuse_courant the Courant maxima are reset by part 1 and complete after
 * part 2. */
int hydro_b200_domain_sweep_part(hb_domain *d, int stage, int idim, double dt, int fuse_courant,
                                 int part);
long long hydro_b200_domain_halo_count(hb_domain *d, int idim);
int hydro_b200_domain_halo_pack(hb_domain *d, int stage, int idim, int side, double *dst);
int hydro_b200_domain_halo_unpack(hb_domain *d, int idim, int side, const double *src);

/* VTK payload of one variable (0..3 = rho, rho u, rho v, E): the interior in
 * row order as floats (C's (float) cast), base64-encoded as vtkfile.c:262-280
 * does, written to host memory; hydro_b200_vtk_base64_len(nx, ny) bytes (no
 * terminator; the 8-character length header is not included). */
long long hydro_b200_vtk_base64_len(int nx, int ny);
int hydro_b200_domain_vtk_base64(hb_domain *d, int var, char *host_out, long long cap);
/* Launch-only driver (asynchronous; same semantics as hydro_b200_run). */
int hydro_b200_domain_set_clock(hb_domain *d, double t, int nstep, double dt);
int hydro_b200_domain_launch_steps(hb_domain *d, int nsteps, int nstepmax, double tend);
int hydro_b200_domain_get_clock(hb_domain *d, double *t, int *nstep, double *dt); /* synchronous */
int hydro_b200_domain_get_dts(hb_domain *d, double *dts, int n); /* dt of the steps since set_clock */
/* Reserve the device record of the dt of up to n steps; set_clock after it
 * starts recording (hydro_b200_run reserves its own). */
int hydro_b200_domain_reserve_dts(hb_domain *d, int n);
/* Arithmetic of the sweeps.  HB_PREC_FP64 (default): the reference's FP64
 * operations, bit for bit.  HB_PREC_MIXED: FP32 constoprim / EOS / slope /
 * trace / Riemann sampling / flux, FP64 Newton iteration on p*, FP64 update
 * and Courant speeds; the state stays FP64.  Mirrors created through the
 * reference entry points use HB_PREC_MIXED when HYDRO_B200_PRECISION=mixed. */
#define HB_PREC_FP64 0
#define HB_PREC_MIXED 1
/* HB_PREC_FP64_FMA: FP64 throughout, with FMA contraction and divisions and
 * square roots through refined reciprocals (one per shared denominator)
 * instead of the reference's IEEE-rounded operations in its order: within
 * 1e-12 of the reference per cell over its 200-step 4096^2 run, not bitwise. */
#define HB_PREC_FP64_FMA 2
int hydro_b200_domain_set_precision(hb_domain *d, int precision);

/* Kernel of the x sweep.  HB_XSWEEP_MARCH: each thread marches along a row
 * segment (as the y sweep does along columns).  HB_XSWEEP_CELL: a warp takes
 * 32 consecutive cells of a row, one per lane, and exchanges neighbours by
 * shuffles (whole-line memory accesses, 28 of 32 lanes productive).  Both give
 * identical results; CELL is the default (faster at 4096^2 for both
 * precisions: the x sweep's loads then use whole lines).  Mirrors
 * created through the reference entry points use HYDRO_B200_XSWEEP=cell|march. */
#define HB_XSWEEP_MARCH 0
#define HB_XSWEEP_CELL 1
int hydro_b200_domain_set_xsweep(hb_domain *d, int precision, int mode);

/* Sweep kernel of one direction (idim 1: x, 2: y) and precision.  All give
 * identical results in FP64; they differ in how lines are cut into work:
 *   HB_KERNEL_MARCH  each thread marches along a line segment with a
 *                    five-cell register window;
 *   HB_KERNEL_WARP   a warp takes 32 consecutive cells of a line, one per lane
 *                    (two per lane in the mixed x sweep), neighbours by warp
 *                    shuffles: 28 outputs per warp (not for the mixed y sweep);
 *   HB_KERNEL_COOP   a CTA of 4 warps takes 128 consecutive cells of a line,
 *                    neighbours through shared memory: 124 outputs per CTA;
 *   HB_KERNEL_COOP8  the same with 8 warps: 252 outputs per CTA;
 *   HB_KERNEL_BULK   mixed x sweep only: runs of two-cell warp windows whose
 *                    cells are staged in shared memory by bulk copies of the
 *                    TMA engine (cp.async.bulk, mbarrier completion) while the
 *                    previous window computes; results identical to
 *                    HB_KERNEL_WARP, whose large-grid form stages by per-lane
 *                    cp.async;
 *   HB_KERNEL_AUTO   the measured default for the grid size.
 * get_kernel returns the current choice (-1 on error). */
#define HB_KERNEL_AUTO (-1)
#define HB_KERNEL_MARCH 0
#define HB_KERNEL_WARP 1
#define HB_KERNEL_COOP 2
#define HB_KERNEL_COOP8 3
#define HB_KERNEL_BULK 4
int hydro_b200_domain_set_kernel(hb_domain *d, int precision, int idim, int kernel);
int hydro_b200_domain_get_kernel(hb_domain *d, int precision, int idim);

/* Event timing of every sweep launch: enable, then read the accumulated
 * milliseconds and launch counts of x (index 0) and y (index 1) sweeps. */
int hydro_b200_domain_profile(hb_domain *d, int enable);
int hydro_b200_domain_profile_read(hb_domain *d, double *ms, long long *count, int reset);
/* Number of kernel launches the library issued on this domain so far. */
long long hydro_b200_domain_launch_count(hb_domain *d);

/* ------------------------------------------------------------------------
 * Batches: many independent runs of different grid sizes advanced together.
 * One global step advances every active instance by one time step of its own
 * (its own dt, main.c:344-408 semantics per instance) with persistent
 * launches (x items and y items of each sweep phase) that pull work items of
 * all instances from a queue; each step is replayed as a CUDA graph.
 * Instance states live in one device arena.
 * ------------------------------------------------------------------------ */
typedef struct hb_batch hb_batch;
/* H supplies the constants shared by every instance (gamma, smallr, smallc,
 * courant_factor, niter_riemann, iorder, slope_type, scheme); capacity is the
 * number of slots, arena_bytes the device memory for states and scratch. */
hb_batch *hydro_b200_batch_create(const hydroparam_t *H, int capacity, size_t arena_bytes,
                                  int precision);
void hydro_b200_batch_destroy(hb_batch *b);
/* Device bytes an instance of grid H takes in the arena. */
long long hydro_b200_batch_bytes_needed(const hydroparam_t *H);
long long hydro_b200_batch_arena_free(hb_batch *b);
/* Admit an instance (grid nx, ny, dx and boundary types from H, clock from
 * H->t and H->nstep, state from host memory in the reference layout); it runs
 * until t >= tend or nstep >= nstepmax.  Returns its slot, or -1 when no slot
 * or arena space is free (HB_ERR_NOMEM). */
int hydro_b200_batch_add(hb_batch *b, const hydroparam_t *H, const double *host, double tend,
                         int nstepmax);
/* Resume a checkpoint (state downloaded with hydro_b200_batch_download, clock
 * read with hydro_b200_batch_status): clock from H->t and H->nstep, and dt,
 * the step size in force (used when H->nstep is odd, as main.c keeps the dt
 * of an even step for the odd step after it). */
int hydro_b200_batch_add_resume(hb_batch *b, const hydroparam_t *H, const double *host, double dt,
                                double tend, int nstepmax);
/* The same with the initial state written on the device: a single blast
 * (density rho, zero momenta, energy e_bg, and e_blast in the padded cell
 * (bi, bj); ghost cells 0). */
int hydro_b200_batch_add_blast(hb_batch *b, const hydroparam_t *H, double rho, double e_bg,
                               int bi, int bj, double e_blast, double tend, int nstepmax);
int hydro_b200_batch_remove(hb_batch *b, int slot);
int hydro_b200_batch_steps(hb_batch *b, int nsteps); /* asynchronous */
int hydro_b200_batch_synchronize(hb_batch *b);
int hydro_b200_batch_status(hb_batch *b, int slot, double *t, int *nstep, double *dt, int *active,
                            long long *stop_step);
int hydro_b200_batch_poll(hb_batch *b, int *active, int n);
/* active / nstep / t of the first n slots in one read (any pointer may be NULL). */
int hydro_b200_batch_table(hb_batch *b, int *active, int *nstep, double *t, int n);
int hydro_b200_batch_download(hb_batch *b, int slot, double *host);
long long hydro_b200_batch_global_step(hb_batch *b);
long long hydro_b200_batch_launch_count(hb_batch *b);
void *hydro_b200_batch_stream(hb_batch *b);
/* Tiling of the work items: y-segment length, items per queue claim,
 * persistent CTAs per SM (0 = occupancy limit), threads per CTA (64 or 128:
 * the columns of a y item; an x item's 8 windows are shared by the CTA's
 * warps).  Results do not depend on it. */
int hydro_b200_batch_set_tuning(hb_batch *b, int seg, int claim, int blocks_per_sm, int threads);
int hydro_b200_batch_get_tuning(hb_batch *b, int *seg, int *claim, int *blocks_per_sm,
                                int *threads);
/* Times `steps` real global steps per candidate tiling and keeps the fastest
 * (cached per mix of grid shapes).  Returns the global steps advanced. */
int hydro_b200_batch_autotune(hb_batch *b, int steps);

/* Select the CUDA device used by the calling thread for domains and mirrors
 * created afterwards (the library links its own CUDA runtime, so a device
 * chosen through another runtime instance does not carry over). */
int hydro_b200_set_device(int device);

/* A hydro_godunov step (FP64, the sweeps of hydro_godunov) for callers that
 * cannot allocate device memory: code running inside another framework's
 * memory arena, which owns the device memory it hands out, or in a process
 * whose device-allocation budget is already spent.  No counterpart in the
 * reference.  The caller holds the state on the device (d_uold, reference
 * layout, 4*(nx+4)*(ny+4) doubles, updated in place) and passes the stream (a
 * cudaStream_t, or NULL).  d_uold must be device or managed memory of the
 * current device (hydro_b200_set_device); anything else, host memory
 * included, is rejected with HB_ERR_ARG.  The second buffer the sweeps need
 * is a static __device__ array of 4*HB_NOALLOC_MAX_CELLS doubles (32 MiB)
 * that every GPU loading the library keeps until exit, so the call makes no
 * cudaMalloc / cudaFree / stream or event creation.  Grids with
 * (nx+4)*(ny+4) > HB_NOALLOC_MAX_CELLS are rejected with HB_ERR_ARG.  It runs
 * the kernels hydro_godunov uses for grids of this size, so the results are
 * the same bits.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the one array: calls whose kernels overlap on
 * the GPU race, so serialise them.  Returns HB_OK or an error code (message
 * in hydro_b200_last_error_message). */
#define HB_NOALLOC_MAX_CELLS (1 << 20)
int hydro_b200_godunov_noalloc(const hydroparam_t *H, double *d_uold, int idim, double dt,
                               void *stream);

/* Library build information (static string). */
const char *hydro_b200_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* HYDRO_B200_H */
