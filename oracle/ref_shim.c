/*
 * ref_shim.c -- ctypes-callable harness around the REFERENCE's own objects.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
 * the reference's unmodified HydroC99_2Domp sources (read in place, never
 * copied) into oracle/_ref/libhydroref.so.  The tests use it to pin the C
 * restatement (oracle/hydro_oracle.c) and the CUDA path against the reference
 * itself; bench.py's reference arm times it.  The product never links it.
 *
 * It mirrors the driver loop of main.c:344-408 and the set-up of
 * main.c:159-244 (process_args defaults from parametres.c:22-71, hydro_init,
 * allocate_work_space, compute_deltat_init_mem) without the I/O.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "parametres.h"
#include "compute_deltat.h"
#include "hydro_funcs.h"
#include "hydro_godunov.h"
#include "make_boundary.h"
#include "vtkfile.h"

#include "orc_param.h"

/* main.c:34 defines the per-stage timers; the driver owns them. */
double functim[TIM_END];

typedef struct {
    hydroparam_t H;
    hydrovar_t Hv;
    hydrowork_t Hw_godunov, Hw_deltat;
    hydrovarwork_t Hvw_godunov, Hvw_deltat;
} ref_state_t;

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* parametres.c:22-71 defaults, then the keys of an .nml file, then the
 * nxystep rule of parametres.c:333-341 and hydro_init. */
void *ref_create(const orc_param_t *P, int testcase, int nxystep) {
    ref_state_t *s = (ref_state_t *)calloc(1, sizeof(ref_state_t));
    hydroparam_t *H = &s->H;
    H->prt = 0;
    H->nproc = 1;
    H->mype = 0;
    H->nvar = IP + 1;
    H->t = 0.0;
    H->nstep = 0;
    H->tend = 0.0;
    H->nstepmax = 0x7fffffff;
    H->shrink = 1;
    H->shrinkSize = 1000;
    H->nx = P->nx;
    H->ny = P->ny;
    H->globnx = P->nx;
    H->globny = P->ny;
    H->box[XMIN_BOX] = 0;
    H->box[XMAX_BOX] = P->nx;
    H->box[YMIN_BOX] = 0;
    H->box[YMAX_BOX] = P->ny;
    H->box[UP_BOX] = H->box[DOWN_BOX] = H->box[LEFT_BOX] = H->box[RIGHT_BOX] = -1;
    H->dx = P->dx;
    H->gamma = P->gamma;
    H->courant_factor = P->courant_factor;
    H->smallc = P->smallc;
    H->smallr = P->smallr;
    H->niter_riemann = P->niter_riemann;
    H->iorder = P->iorder;
    H->slope_type = P->slope_type;
    H->scheme = P->scheme;
    H->boundary_left = P->boundary_left;
    H->boundary_right = P->boundary_right;
    H->boundary_down = P->boundary_down;
    H->boundary_up = P->boundary_up;
    H->testCase = testcase;
    H->nxystep = nxystep;
    if (H->nxystep <= 0) {
        H->nxystep = (H->nx < H->ny) ? H->nx : H->ny;
    } else {
        if (H->nxystep > H->nx) H->nxystep = H->nx;
        if (H->nxystep > H->ny) H->nxystep = H->ny;
    }
    hydro_init(H, &s->Hv);
    allocate_work_space(H->nxyt, *H, &s->Hw_godunov, &s->Hvw_godunov);
    compute_deltat_init_mem(*H, &s->Hw_deltat, &s->Hvw_deltat);
    return s;
}

void ref_destroy(void *h) {
    ref_state_t *s = (ref_state_t *)h;
    deallocate_work_space(s->H.nxyt, s->H, &s->Hw_godunov, &s->Hvw_godunov);
    compute_deltat_clean_mem(s->H, &s->Hw_deltat, &s->Hvw_deltat);
    hydro_finish(s->H, &s->Hv);
    free(s);
}

long ref_ncells(void *h) {
    ref_state_t *s = (ref_state_t *)h;
    return (long)s->H.nvar * s->H.nxt * s->H.nyt;
}

/* The state crosses the harness as doubles whatever real_t is (the single-
 * precision build, -DPREC_SP, converts on the way in and out). */
void ref_get(void *h, double *out) {
    ref_state_t *s = (ref_state_t *)h;
    const long n = ref_ncells(h);
    for (long i = 0; i < n; i++) out[i] = (double)s->Hv.uold[i];
}

void ref_set(void *h, const double *in) {
    ref_state_t *s = (ref_state_t *)h;
    const long n = ref_ncells(h);
    for (long i = 0; i < n; i++) s->Hv.uold[i] = (real_t)in[i];
}

double ref_compute_deltat(void *h) {
    ref_state_t *s = (ref_state_t *)h;
    real_t dt = 0;
    compute_deltat(&dt, s->H, &s->Hw_deltat, &s->Hv, &s->Hvw_deltat);
    return dt;
}

void ref_godunov(void *h, int idim, double dt) {
    ref_state_t *s = (ref_state_t *)h;
    hydro_godunov(idim, dt, s->H, &s->Hv, &s->Hw_godunov, &s->Hvw_godunov);
}

void ref_make_boundary(void *h, int idim) {
    ref_state_t *s = (ref_state_t *)h;
    make_boundary(idim, s->H, &s->Hv);
}

/* main.c:344-408.  Runs until t >= tend or nstep >= nstepmax counted from the
 * state's current (t, nstep).  dts (optional) receives each step's dt.
 * mcs_avg receives the reference's "Average MC/s" statistic (main.c:485-513:
 * mean of the per-step MC/s over steps with nstep > 5); elapsed the wall time. */
int ref_run(void *h, int nstepmax, double tend, double *dts, double *t_out, double *mcs_avg,
            double *elapsed) {
    ref_state_t *s = (ref_state_t *)h;
    hydroparam_t *H = &s->H;
    real_t dt = 0;
    double sum = 0;
    long nsum = 0;
    int n0 = H->nstep;
    double t_start = now_s();
    while ((H->t < tend) && (H->nstep < nstepmax)) {
        double t0 = now_s();
        if ((H->nstep % 2) == 0) {
            dt = 0;
            compute_deltat(&dt, *H, &s->Hw_deltat, &s->Hv, &s->Hvw_deltat);
            if (H->nstep == 0) dt = dt / 2.0;
        }
        if ((H->nstep % 2) == 0)
            hydro_godunov(1, dt, *H, &s->Hv, &s->Hw_godunov, &s->Hvw_godunov);
        else
            hydro_godunov(2, dt, *H, &s->Hv, &s->Hw_godunov, &s->Hvw_godunov);
        double t1 = now_s();
        if (dts) dts[H->nstep - n0] = dt;
        H->nstep++;
        H->t += dt;
        double mcs = (double)H->globnx * H->globny / (t1 - t0) / 1e6;
        if (H->nstep > 5) {
            sum += mcs;
            nsum++;
        }
    }
    if (t_out) *t_out = H->t;
    if (mcs_avg) *mcs_avg = nsum ? sum / nsum : 0.0;
    if (elapsed) *elapsed = now_s() - t_start;
    return H->nstep - n0;
}

/* real_t of this build: 8 (double) or 4 (-DPREC_SP). */
int ref_real_size(void) { return (int)sizeof(real_t); }

/* Struct layout of hydroparam_t as the reference compiles it: size and the
 * offset of every field, for the ABI-compatibility test of include/. */
#include <stddef.h>
#define OFF(f) (long)offsetof(hydroparam_t, f)
int ref_param_layout(long *out, int nmax) {
    long v[] = {(long)sizeof(hydroparam_t), OFF(prt), OFF(t), OFF(tend), OFF(nstep),
                OFF(nstepmax), OFF(noutput), OFF(dtoutput), OFF(nimage), OFF(dtimage),
                OFF(imin), OFF(imax), OFF(jmin), OFF(jmax), OFF(nx), OFF(ny), OFF(nxt),
                OFF(nyt), OFF(nxyt), OFF(nxystep), OFF(nproc), OFF(mype), OFF(globnx),
                OFF(globny), OFF(box), OFF(nvar), OFF(dx), OFF(gamma), OFF(courant_factor),
                OFF(smallc), OFF(smallr), OFF(niter_riemann), OFF(iorder), OFF(slope_type),
                OFF(scheme), OFF(boundary_right), OFF(boundary_left), OFF(boundary_down),
                OFF(boundary_up), OFF(testCase), OFF(shrinkSize), OFF(shrink), OFF(fp),
                (long)sizeof(hydrovar_t), (long)sizeof(hydrowork_t),
                (long)sizeof(hydrovarwork_t)};
    int n = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < nmax; i++) out[i] = v[i];
    return n;
}

/* The reference's own parameter reader (parametres.c:230-357) on an .nml
 * file; copies the fields the C ABI consumes into out[] in this order:
 * nx ny nxystep nstepmax iorder niter_riemann scheme boundary_left
 * boundary_right boundary_down boundary_up testCase (ints, as doubles)
 * tend dx courant_factor smallr smallc slope_type gamma. */
int ref_parse_nml(const char *path, double *out) {
    hydroparam_t H;
    char a0[] = "hydro", a1[] = "-i";
    char a2[512];
    strncpy(a2, path, sizeof(a2) - 1);
    a2[sizeof(a2) - 1] = 0;
    char *argv[] = {a0, a1, a2, NULL};
    memset(&H, 0, sizeof(H));
    process_args(3, argv, &H);
    double v[] = {H.nx, H.ny, H.nxystep, H.nstepmax, H.iorder, H.niter_riemann, H.scheme,
                  H.boundary_left, H.boundary_right, H.boundary_down, H.boundary_up, H.testCase,
                  H.tend, H.dx, H.courant_factor, H.smallr, H.smallc, H.slope_type, H.gamma};
    int n = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n; i++) out[i] = v[i];
    return n;
}

/* The reference's VTK writer (vtkfile.c:140-352) on the state, into the
 * current directory; output number `step`. */
void ref_vtkfile(void *h, int step) {
    ref_state_t *s = (ref_state_t *)h;
    vtkfile(step, s->H, &s->Hv);
}
