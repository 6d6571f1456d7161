/*
 * hydro_oracle.c -- CPU restatement of the HydroC99_2Domp time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only
 * the test-suite, the smoke check and bench.py's CPU-baseline leg load it.  The
 * product library (hydro_b200/csrc) never includes, links or calls it.
 *
 * It restates, line by line of arithmetic, the reference algorithm in
 * HydroC/HydroC99_2Domp/Src (all citations below are relative to that
 * directory).  The reference processes "strips" of nxystep rows/columns with
 * work arrays u,q,dq,qxm,... (hydro_godunov.c:106-138); this restatement
 * processes one line (a row for the x sweep, a column for the y sweep) at a
 * time, which the reference shows to be equivalent: every stage is pointwise
 * along the line and lines are independent.  Each IEEE operation is written in
 * the same order as the reference so the result is bitwise identical to the
 * reference built without FMA contraction (checked by tests/test_oracle.py
 * against the reference itself and against tests/golden).
 *
 * State layout (parametres.h:92-93): uold[v][j][i], index i + nxt*(j + nyt*v),
 * nxt = nx+4, nyt = ny+4, v in {ID=0 rho, IU=1 rho*u, IV=2 rho*v, IP=3 E}.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "orc_param.h"

enum { ID = 0, IU = 1, IV = 2, IP = 3, NV = 4, XL = 2 };

/* MAX macro of utils.h:9-11 (not fmax: NaN and tie behaviour differ). */
#define OMAX(x, y) ((x) > (y) ? (x) : (y))

static inline long cell(const orc_param_t *P, int i, int j, int v) {
    long nxt = P->nx + 4, nyt = P->ny + 4;
    return i + nxt * (j + nyt * (long)v);
}

/* hydro_funcs.c:15-112 with nproc == 1: interior rho=1,u=v=0,E=1e-5, ghosts 0,
 * blast E = one/dx/dx at the padded centre (0), corner (2,2) (1) or the column
 * x=2 from j=2 to jmax-1 (2). */
int orc_init(const orc_param_t *P, int testcase, double *uold) {
    int nxt = P->nx + 4, nyt = P->ny + 4;
    memset(uold, 0, sizeof(double) * (size_t)NV * nxt * nyt);
    for (int j = XL; j < nyt - XL; j++)
        for (int i = XL; i < nxt - XL; i++) {
            uold[cell(P, i, j, ID)] = 1.0;
            uold[cell(P, i, j, IU)] = 0.0;
            uold[cell(P, i, j, IV)] = 0.0;
            uold[cell(P, i, j, IP)] = 1e-5;
        }
    double eblast = 1.0 / P->dx / P->dx;
    if (testcase == 0) {
        uold[cell(P, nxt / 2, nyt / 2, IP)] = eblast;
    } else if (testcase == 1) {
        uold[cell(P, XL, XL, IP)] = eblast;
    } else if (testcase == 2) {
        for (int j = XL; j < nyt; j++) uold[cell(P, XL, j, IP)] = eblast;
    } else {
        return -1;
    }
    return 0;
}

/* make_boundary.c:53-198.  Ghost source index and sign for one side. */
static void ghost_src(int btype, int side_low, int k, int nlen, int *src) {
    /* k: ghost position along the line (0,1 low side; nlen+2,nlen+3 high side).
     * nlen: nx or ny. */
    if (side_low) {
        if (btype == 1) *src = 2 * XL - k - 1;         /* make_boundary.c:63-67 */
        else if (btype == 2) *src = 2;                 /* :68-69 ("absorb")     */
        else *src = nlen + k;                          /* :70-71 (periodic)     */
    } else {
        if (btype == 1) *src = 2 * nlen + 2 * XL - k - 1; /* :98-102 */
        else if (btype == 2) *src = nlen + XL;            /* :103-104 */
        else *src = k - nlen;                             /* :105-106 */
    }
}

void orc_make_boundary(const orc_param_t *P, int idim, double *uold) {
    int nx = P->nx, ny = P->ny;
    if (idim == 1) {
        if (P->boundary_left > 0)
            for (int v = 0; v < NV; v++)
                for (int k = 0; k < XL; k++) {
                    int src;
                    ghost_src(P->boundary_left, 1, k, nx, &src);
                    double sign = (P->boundary_left == 1 && v == IU) ? -1.0 : 1.0;
                    for (int j = XL; j < ny + XL; j++)
                        uold[cell(P, k, j, v)] = uold[cell(P, src, j, v)] * sign;
                }
        if (P->boundary_right > 0)
            for (int v = 0; v < NV; v++)
                for (int k = nx + XL; k < nx + 2 * XL; k++) {
                    int src;
                    ghost_src(P->boundary_right, 0, k, nx, &src);
                    double sign = (P->boundary_right == 1 && v == IU) ? -1.0 : 1.0;
                    for (int j = XL; j < ny + XL; j++)
                        uold[cell(P, k, j, v)] = uold[cell(P, src, j, v)] * sign;
                }
    } else {
        if (P->boundary_down > 0)
            for (int v = 0; v < NV; v++)
                for (int k = 0; k < XL; k++) {
                    int src;
                    if (P->boundary_down == 1) src = 2 * XL - k - 1;   /* :140-144 */
                    else if (P->boundary_down == 2) src = 2 * XL;      /* :145-146 */
                    else src = ny + k;                                 /* :147-148 */
                    double sign = (P->boundary_down == 1 && v == IV) ? -1.0 : 1.0;
                    for (int i = XL; i < nx + XL; i++)
                        uold[cell(P, i, k, v)] = uold[cell(P, i, src, v)] * sign;
                }
        if (P->boundary_up > 0)
            for (int v = 0; v < NV; v++)
                for (int k = ny + XL; k < ny + 2 * XL; k++) {
                    int src;
                    if (P->boundary_up == 1) src = 2 * ny + 2 * XL - k - 1; /* :176-180 */
                    else if (P->boundary_up == 2) src = ny + 1;             /* :181-182 */
                    else src = k - ny;                                      /* :183-184 */
                    double sign = (P->boundary_up == 1 && v == IV) ? -1.0 : 1.0;
                    for (int i = XL; i < nx + XL; i++)
                        uold[cell(P, i, k, v)] = uold[cell(P, i, src, v)] * sign;
                }
    }
}

typedef struct { double r, u, v, p; } prim4;

/* constoprim.c:37-52 followed by equation_of_state.c:41-48. */
static inline void cons_to_prim(const orc_param_t *P, double d, double mn, double mt, double en,
                                prim4 *q, double *c) {
    double smallp = (P->smallc * P->smallc) / P->gamma; /* equation_of_state.c:25 */
    double r = OMAX(d, P->smallr);
    double un = mn / r;
    double ut = mt / r;
    double eken = 0.5 * ((un * un) + (ut * ut));
    double e = en / r - eken;
    double base = (P->gamma - 1.0) * r * e;
    base = OMAX(base, (double)(r * smallp));
    q->r = r;
    q->u = un;
    q->v = ut;
    q->p = base;
    *c = sqrt(P->gamma * base / r);
}

/* slope.c:37-50, one variable. */
static inline double slope1(double st, double qm, double q0, double qp) {
    double dlft = st * (q0 - qm);
    double drgt = st * (qp - q0);
    double dcen = 0.5 * (dlft + drgt) / st;
    double dsgn = (dcen > 0.0) ? 1.0 : -1.0;
    int llftrgt = ((dlft * drgt) <= 0.0);
    double t1 = fmin(fabs(dlft), fabs(drgt));
    return dsgn * fmin((double)(1 - llftrgt) * t1, fabs(dcen));
}

/* trace.c:30-46 (scheme constants) and :63-123 (per cell). */
static inline void trace1(double dtdx, double zerol, double zeror, double project, prim4 q,
                          prim4 dq, double cc, prim4 *qxm, prim4 *qxp) {
    double csq = cc * cc;
    double r = q.r, u = q.u, v = q.v, p = q.p;
    double dr = dq.r, du = dq.u, dv = dq.v, dp = dq.p;
    double rOcc = r / cc;
    double OrOcc = cc / r;
    double dprcc = dp / (r * cc);
    double alpham = 0.5 * (dprcc - du) * rOcc;
    double alphap = 0.5 * (dprcc + du) * rOcc;
    double alpha0r = dr - dp / csq;
    double alpha0v = dv;
    double upcc = u + cc;
    double umcc = u - cc;
    double upccx = upcc * dtdx;
    double umccx = umcc * dtdx;
    double ux = u * dtdx;

    double spminus = (umcc >= zeror) ? (project) : umccx + 1.0;
    double spplus = (upcc >= zeror) ? (project) : upccx + 1.0;
    double spzero = (u >= zeror) ? (project) : ux + 1.0;
    double ap = -0.5 * spplus * alphap;
    double am = -0.5 * spminus * alpham;
    double azr = -0.5 * spzero * alpha0r;
    double azv = -0.5 * spzero * alpha0v;
    qxp->r = r + (ap + am + azr);
    qxp->u = u + (ap - am) * OrOcc;
    qxp->v = v + (azv);
    qxp->p = p + (ap + am) * csq;

    spminus = (umcc <= zerol) ? (-project) : umccx - 1.0;
    spplus = (upcc <= zerol) ? (-project) : upccx - 1.0;
    spzero = (u <= zerol) ? (-project) : ux - 1.0;
    ap = -0.5 * spplus * alphap;
    am = -0.5 * spminus * alpham;
    azr = -0.5 * spzero * alpha0r;
    azv = -0.5 * spzero * alpha0v;
    qxm->r = r + (ap + am + azr);
    qxm->u = u + (ap - am) * OrOcc;
    qxm->v = v + (azv);
    qxm->p = p + (ap + am) * csq;
}

/* riemann.c:89-110 (first guess), :126-156 (Newton on p*), :175-258 (sampling,
 * C99 selection order: outer state if spout<0, else star if spin>0, else
 * blend), then cmpflx.c:52-73 (flux of the Godunov state). */
static inline void riemann_flux(const orc_param_t *P, prim4 ql, prim4 qr, double f[4]) {
    const double gamma = P->gamma, smallr = P->smallr, smallc = P->smallc;
    double smallp = (smallc * smallc) / gamma;
    double gamma6 = (gamma + 1.0) / (2.0 * gamma);
    double smallpp = smallr * smallp;

    double rl = fmax(ql.r, smallr);
    double ul = ql.u;
    double pl = fmax(ql.p, (double)(rl * smallp));
    double rr = fmax(qr.r, smallr);
    double ur = qr.u;
    double pr = fmax(qr.p, (double)(rr * smallp));
    double cl = gamma * pl * rl;
    double cr = gamma * pr * rr;
    double wl = sqrt(cl);
    double wr = sqrt(cr);
    double pstar = fmax(((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr), 0.0);

    for (int iter = 0; iter < P->niter_riemann; iter++) {
        double pst = pstar;
        double wwl = sqrt(cl * (1.0 + gamma6 * (pst - pl) / pl));
        double wwr = sqrt(cr * (1.0 + gamma6 * (pst - pr) / pr));
        double swwl = wwl * wwl;
        double qlw = 2.0 * wwl * swwl / (swwl + cl);
        double qrw = 2.0 * wwr * (wwr * wwr) / ((wwr * wwr) + cr);
        double usl = ul - (pst - pl) / wwl;
        double usr = ur + (pst - pr) / wwr;
        double tmp = (qrw * qlw / (qrw + qlw) * (usl - usr));
        double delp = OMAX(tmp, (-pst));
        pst += delp;
        double tmp2 = delp / (pst + smallpp);
        double conv = fabs(tmp2);
        pstar = pst;
        if (!(conv > 1e-6)) break; /* goon[] mask of riemann.c:131,153 */
    }

    wr = sqrt(cr * (1.0 + gamma6 * (pstar - pr) / pr));
    wl = sqrt(cl * (1.0 + gamma6 * (pstar - pl) / pl));
    double ustar = 0.5 * (ul + (pl - pstar) / wl + ur - (pr - pstar) / wr);
    int left = ustar > 0;
    int sgnm = left ? 1 : -1;
    double ro = left ? rl : rr;
    double uo = left ? ul : ur;
    double po = left ? pl : pr;
    double wo = left ? wl : wr;
    double co = sqrt(fabs(gamma * po / ro));
    co = fmax(smallc, co);
    double rstar = ro / (1.0 + ro * (po - pstar) / (wo * wo));
    rstar = fmax(rstar, smallr);
    double cstar = sqrt(fabs(gamma * pstar / rstar));
    cstar = fmax(smallc, cstar);
    double spout = co - sgnm * uo;
    double spin = cstar - sgnm * ustar;
    double ushock = wo / ro - sgnm * uo;
    if (pstar >= po) {
        spin = ushock;
        spout = ushock;
    }
    double scr = fmax((double)(spout - spin), (double)(smallc + fabs(spout + spin)));
    double frac = (1.0 + (spout + spin) / scr) * 0.5;
    frac = fmax(0.0, (double)(fmin(1.0, frac)));
    double gr, gu, gp;
    if (spout < 0.0) {
        gr = ro; gu = uo; gp = po;
    } else if (spin > 0.0) {
        gr = rstar; gu = ustar; gp = pstar;
    } else {
        gr = (frac * rstar + (1.0 - frac) * ro);
        gu = (frac * ustar + (1.0 - frac) * uo);
        gp = (frac * pstar + (1.0 - frac) * po);
    }
    double gv = left ? ql.v : qr.v;

    double entho = 1.0 / (gamma - 1.0); /* cmpflx.c:27 */
    double mass = gr * gu;
    f[0] = mass;
    f[1] = mass * gu + gp;
    f[2] = mass * gv;
    double ekin = 0.5 * gr * ((gu * gu) + (gv * gv));
    double etot = gp * entho + ekin;
    f[3] = gu * (etot + gp);
}

/* One line of one sweep: gatherConservativeVars (conservar.c:40-56, y with the
 * IU<->IV swap of :97-100), constoprim, equation_of_state, slope, trace,
 * qleftright (qleftright.c:41-50), riemann, cmpflx and
 * updateConservativeVars (conservar.c:166-172, y: :207-218). */
static void sweep_line(const orc_param_t *P, int idim, int line, double dtdx, double *uold,
                       double *work, int n) {
    double *cons = work;              /* [4][n] */
    prim4 *q = (prim4 *)(cons + 4 * n);
    double *c = (double *)(q + n);
    prim4 *dq = (prim4 *)(c + n);
    prim4 *qxm = dq + n;
    prim4 *qxp = qxm + n;
    double *flux = (double *)(qxp + n); /* [n][4] */
    int nface = (idim == 1 ? P->nx : P->ny) + 1;
    int mn = (idim == 1) ? IU : IV, mt = (idim == 1) ? IV : IU;

    for (int k = 0; k < n; k++) {
        long b = (idim == 1) ? cell(P, k, line, 0) : cell(P, line, k, 0);
        long vs = (long)(P->nx + 4) * (P->ny + 4);
        cons[0 * n + k] = uold[b + ID * vs];
        cons[1 * n + k] = uold[b + mn * vs];
        cons[2 * n + k] = uold[b + mt * vs];
        cons[3 * n + k] = uold[b + IP * vs];
        cons_to_prim(P, cons[k], cons[n + k], cons[2 * n + k], cons[3 * n + k], &q[k], &c[k]);
    }
    memset(dq, 0, sizeof(prim4) * n);
    if (P->iorder != 1) {
        for (int k = 1; k < n - 1; k++) {
            dq[k].r = slope1(P->slope_type, q[k - 1].r, q[k].r, q[k + 1].r);
            dq[k].u = slope1(P->slope_type, q[k - 1].u, q[k].u, q[k + 1].u);
            dq[k].v = slope1(P->slope_type, q[k - 1].v, q[k].v, q[k + 1].v);
            dq[k].p = slope1(P->slope_type, q[k - 1].p, q[k].p, q[k + 1].p);
        }
    }
    double zerol = 0.0, zeror = 0.0, project = 0.0;
    if (P->scheme == 1) { zerol = -100.0 / dtdx; zeror = 100.0 / dtdx; project = 1.0; }
    if (P->scheme == 2) { zerol = 0.0; zeror = 0.0; project = 1.0; }
    if (P->scheme == 3) { zerol = 0.0; zeror = 0.0; project = 0.0; }
    for (int k = 1; k < n - 1; k++)
        trace1(dtdx, zerol, zeror, project, q[k], dq[k], c[k], &qxm[k], &qxp[k]);
    for (int m = 0; m < nface; m++) riemann_flux(P, qxm[m + 1], qxp[m + 2], &flux[4 * m]);
    for (int k = XL; k < n - XL; k++) {
        long b = (idim == 1) ? cell(P, k, line, 0) : cell(P, line, k, 0);
        long vs = (long)(P->nx + 4) * (P->ny + 4);
        int slot[4] = {ID, mn, mt, IP};
        for (int v = 0; v < 4; v++)
            uold[b + slot[v] * vs] =
                cons[v * n + k] + (flux[4 * (k - 2) + v] - flux[4 * (k - 1) + v]) * dtdx;
    }
}

/* One sweep of hydro_godunov.c:74-139: make_boundary for direction idim, then
 * every line of that direction. */
void orc_sweep(const orc_param_t *P, int idim, double dt, double *uold) {
    int nmax = (P->nx > P->ny ? P->nx : P->ny) + 4;
    double dtdx = dt / P->dx;
    orc_make_boundary(P, idim, uold);
    int nlines = (idim == 1) ? P->ny : P->nx;
    int n = (idim == 1) ? P->nx + 4 : P->ny + 4;
#pragma omp parallel
    {
        double *work = (double *)malloc(sizeof(double) * 4 * 8 * (size_t)nmax + 64);
#pragma omp for schedule(static)
        for (int l = 0; l < nlines; l++) sweep_line(P, idim, l + XL, dtdx, uold, work, n);
        free(work);
    }
}

/* hydro_godunov.c:70-139: two sweeps, order x->y for idim 1, y->x for 2. */
void orc_godunov(const orc_param_t *P, int idimStart, double dt, double *uold) {
    for (int ii = 0; ii < 2; ii++) orc_sweep(P, (idimStart - 1 + ii) % 2 + 1, dt, uold);
}

/* compute_deltat.c:31-77 with ComputeQEforRow.c:31-47, equation_of_state.c
 * and courantOnXY.c:34-47.  Returns dt; stores the two Courant maxima. */
double orc_courant(const orc_param_t *P, const double *uold, double *cx_out, double *cy_out) {
    double cx = 0.0, cy = 0.0;
    for (int j = XL; j < P->ny + XL; j++)
        for (int i = XL; i < P->nx + XL; i++) {
            prim4 q;
            double c;
            double d = uold[cell(P, i, j, ID)];
            double mu = uold[cell(P, i, j, IU)];
            double mv = uold[cell(P, i, j, IV)];
            double en = uold[cell(P, i, j, IP)];
            cons_to_prim(P, d, mu, mv, en, &q, &c);
            cx = OMAX(cx, c + fabs(q.u));
            cy = OMAX(cy, c + fabs(q.v));
        }
    if (cx_out) *cx_out = cx;
    if (cy_out) *cy_out = cy;
    return P->courant_factor * P->dx / OMAX(cx, OMAX(cy, P->smallc));
}

/* main.c:344-408: dt recomputed on even steps, halved at step 0; x->y on even
 * steps, y->x on odd steps.  Returns the number of steps; dts[] gets each
 * step's dt (if not NULL, length >= nstepmax). */
int orc_run(const orc_param_t *P, double *uold, int nstepmax, double tend, double *dts,
            double *t_out) {
    double t = 0.0, dt = 0.0;
    int nstep = 0;
    while (t < tend && nstep < nstepmax) {
        if (nstep % 2 == 0) {
            dt = orc_courant(P, uold, NULL, NULL);
            if (nstep == 0) dt = dt / 2.0;
        }
        orc_godunov(P, (nstep % 2 == 0) ? 1 : 2, dt, uold);
        if (dts) dts[nstep] = dt;
        nstep++;
        t += dt;
    }
    if (t_out) *t_out = t;
    return nstep;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}
