// hb_stages.cuh -- per-cell / per-interface device functions of the HydroC
// Godunov/MUSCL step, FP64.
//
// Every function restates the arithmetic of the reference
// (HydroC/HydroC99_2Domp/Src, cited per function) with the same IEEE
// operations in the same order.  The translation unit that includes this file
// is compiled with --fmad=false and IEEE division / square root, so each
// operation is rounded once, exactly as in the reference's C build (gcc -O3
// -mavx2, no FMA): the kernels reproduce the reference bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hb {

// Primitive variables of one cell in line orientation: density, velocity
// normal to the sweep, transverse velocity, pressure.
struct Prim {
    double r, u, v, p;
};

// Conservative variables in line orientation: rho, normal momentum,
// transverse momentum, total energy.
struct Cons {
    double d, mn, mt, e;
};

// Constants of one run, derived on the host with the reference's formulas.
struct Phys {
    double gamma, gm1;    // gamma, gamma - 1 (equation_of_state.c:42)
    double smallr, smallc;
    double smallp;        // smallc^2 / gamma (equation_of_state.c:25, riemann.c:34)
    double gamma6;        // (gamma + 1) / (2 gamma) (riemann.c:35)
    double smallpp;       // smallr * smallp (riemann.c:36)
    double entho;         // 1 / (gamma - 1) (cmpflx.c:27)
    double slope_type;
    double dx;
    int niter;            // niter_riemann
    int iorder;           // 1: first order (dq = 0)
    int scheme;           // 1 muscl, 2 plmde, 3 collela
    int unit_slope;       // slope_type == 1.0 (x*1 and x/1 are exact: skipped)
};

// utils.h:9-11 MAX(x, y): x > y ? x : y.
__device__ __forceinline__ double omax(double x, double y) { return x > y ? x : y; }

// C99 fmax / fmin as glibc evaluates them for non-NaN operands: x when
// x >= y (resp. x <= y), so a tie between +0 and -0 returns the first operand,
// which PTX max.f64/min.f64 do not promise.  (NaN operands, which a valid
// state never produces, are not given C99's "return the other operand" rule.)
__device__ __forceinline__ double cfmax(double x, double y) { return x >= y ? x : y; }
__device__ __forceinline__ double cfmin(double x, double y) { return x <= y ? x : y; }

// a / b, IEEE-rounded, for a denominator b that is finite and nonzero (every
// call site divides by a positive quantity of a valid state).  A zero
// numerator gives its signed zero as the product a * b, which has the
// quotient's sign and value, without entering the division: the IEEE division
// sequence sends a zero numerator down its slow path (a called subroutine),
// and a cell at rest (zero velocities, uniform pressure) meets 14 such
// numerators per sweep.  Nonzero numerators take the ordinary division, so
// the result is bitwise a / b in every case.
__device__ __forceinline__ double zdiv(double a, double b) {
    if (a == 0.0) return a * b;
    return a / b;
}

// sqrt(x) for an x that often equals x0 > 0 whose square root r0 is already
// known (a Riemann problem between equal states has c_r == c_l, and evaluates
// W = sqrt(c (1 + 0)) four times with the c of its first guess): x == x0 means
// the same bits, so r0 is sqrt(x) exactly.
__device__ __forceinline__ double sqrt_eq(double x, double x0, double r0) {
    if (x == x0) return r0;
    return sqrt(x);
}

// a / b for a b that is often exactly 1 (rho* = rho_o / (1 + 0) between equal
// states): a / 1 is a.
__device__ __forceinline__ double div1(double a, double b) {
    if (b == 1.0) return a;
    return a / b;
}

// constoprim.c:37-52 then equation_of_state.c:41-48.
__device__ __forceinline__ void cons_to_prim(const Phys& P, const Cons& u, Prim& q, double& c) {
    double r = omax(u.d, P.smallr);
    double un = zdiv(u.mn, r);
    double ut = zdiv(u.mt, r);
    double eken = 0.5 * ((un * un) + (ut * ut));
    double e = u.e / r - eken;
    double base = P.gm1 * r * e;
    base = omax(base, r * P.smallp);
    q.r = r;
    q.u = un;
    q.v = ut;
    q.p = base;
    c = sqrt(P.gamma * base / r);
}

// slope.c:37-50 for one variable.
template <bool UNIT>
__device__ __forceinline__ double slope1(double st, double qm, double q0, double qp) {
    double dlft, drgt, dcen;
    if (UNIT) {
        dlft = q0 - qm;
        drgt = qp - q0;
        dcen = 0.5 * (dlft + drgt);
    } else {
        dlft = st * (q0 - qm);
        drgt = st * (qp - q0);
        dcen = 0.5 * (dlft + drgt) / st;
    }
    // dsgn * fmin((1 - llftrgt) * t1, |dcen|) of the reference, written as a
    // select: for finite slopes (1 - llftrgt) * t1 is t1 or +0, fmin(+0, x >= 0)
    // is +0, and (-1) * m is -m exactly, so the bits are the same.
    const bool llftrgt = (dlft * drgt) <= 0.0;
    const double t1 = cfmin(fabs(dlft), fabs(drgt));
    const double m = llftrgt ? 0.0 : cfmin(t1, fabs(dcen));
    return (dcen > 0.0) ? m : -m;
}

// A flat neighbourhood (every variable's two differences exactly zero, which
// also excludes infinities) gives -0 for every slope: +0 differences, +0
// centred slope, a limited magnitude of +0 and the negative branch of the
// sign select, the same bits slope1 computes.
__device__ __forceinline__ bool flat3(const Prim& a, const Prim& b, const Prim& c) {
    return b.r - a.r == 0.0 && c.r - b.r == 0.0 && b.u - a.u == 0.0 && c.u - b.u == 0.0 &&
           b.v - a.v == 0.0 && c.v - b.v == 0.0 && b.p - a.p == 0.0 && c.p - b.p == 0.0;
}

template <bool UNIT>
__device__ __forceinline__ void slope4(double st, const Prim& a, const Prim& b, const Prim& c,
                                       Prim& dq) {
    if (flat3(a, b, c)) {
        dq = Prim{-0.0, -0.0, -0.0, -0.0};
        return;
    }
    dq.r = slope1<UNIT>(st, a.r, b.r, c.r);
    dq.u = slope1<UNIT>(st, a.u, b.u, c.u);
    dq.v = slope1<UNIT>(st, a.v, b.v, c.v);
    dq.p = slope1<UNIT>(st, a.p, b.p, c.p);
}

// Scheme constants of trace.c:30-46.
struct TraceK {
    double dtdx, zerol, zeror, project;
};

__device__ __forceinline__ TraceK trace_constants(int scheme, double dtdx) {
    TraceK k;
    k.dtdx = dtdx;
    k.zerol = 0.0;
    k.zeror = 0.0;
    k.project = 0.0;
    if (scheme == 1) {
        k.zerol = -100.0 / dtdx;
        k.zeror = 100.0 / dtdx;
        k.project = 1.0;
    }
    if (scheme == 2) {
        k.project = 1.0;
    }
    return k;
}

// trace.c:63-123 for one cell: left (qxm) and right (qxp) states.
__device__ __forceinline__ void trace1(const TraceK& K, const Prim& q, const Prim& dq, double cc,
                                       Prim& qxm, Prim& qxp) {
    const double dtdx = K.dtdx;
    // With every slope zero (of either sign), the four factors below only scale
    // signed zeros, and any positive finite factor gives those zeros the same
    // signs: such a cell (the flat cells of a state at rest, or extrema) takes 1
    // for each and skips both IEEE divisions, with the same bits.  The range
    // test keeps the general factors finite and nonzero where this is taken.
    const bool zero_slopes = dq.r == 0.0 && dq.u == 0.0 && dq.v == 0.0 && dq.p == 0.0 &&
                             cc > 1e-100 && cc < 1e100 && q.r > 1e-100 && q.r < 1e100;
    double csq = 1.0, rOcc = 1.0, OrOcc = 1.0, rcc = 1.0;
    if (!zero_slopes) {
        csq = cc * cc;
        rOcc = q.r / cc;
        OrOcc = cc / q.r;
        rcc = q.r * cc;
    }
    double dprcc = zdiv(dq.p, rcc);
    double alpham = 0.5 * (dprcc - dq.u) * rOcc;
    double alphap = 0.5 * (dprcc + dq.u) * rOcc;
    double alpha0r = dq.r - zdiv(dq.p, csq);
    double alpha0v = dq.v;
    double upcc = q.u + cc;
    double umcc = q.u - cc;
    double upccx = upcc * dtdx;
    double umccx = umcc * dtdx;
    double ux = q.u * dtdx;

    double spminus = (umcc >= K.zeror) ? (K.project) : umccx + 1.0;
    double spplus = (upcc >= K.zeror) ? (K.project) : upccx + 1.0;
    double spzero = (q.u >= K.zeror) ? (K.project) : ux + 1.0;
    double ap = -0.5 * spplus * alphap;
    double am = -0.5 * spminus * alpham;
    double azr = -0.5 * spzero * alpha0r;
    double azv = -0.5 * spzero * alpha0v;
    qxp.r = q.r + (ap + am + azr);
    qxp.u = q.u + (ap - am) * OrOcc;
    qxp.v = q.v + (azv);
    qxp.p = q.p + (ap + am) * csq;

    spminus = (umcc <= K.zerol) ? (-K.project) : umccx - 1.0;
    spplus = (upcc <= K.zerol) ? (-K.project) : upccx - 1.0;
    spzero = (q.u <= K.zerol) ? (-K.project) : ux - 1.0;
    ap = -0.5 * spplus * alphap;
    am = -0.5 * spminus * alpham;
    azr = -0.5 * spzero * alpha0r;
    azv = -0.5 * spzero * alpha0v;
    qxm.r = q.r + (ap + am + azr);
    qxm.u = q.u + (ap - am) * OrOcc;
    qxm.v = q.v + (azv);
    qxm.p = q.p + (ap + am) * csq;
}

// riemann.c:89-110 (first guess), :126-156 (Newton iterations on p*, at most
// niter, stopping per interface once |dp/p| <= 1e-6), :175-258 (sampling, with
// the C99 selection order: outer state if spout < 0, else star state if
// spin > 0, else the blend), then the flux of the Godunov state
// (cmpflx.c:52-73).  ql = qxm of the cell left of the interface, qr = qxp of
// the cell to its right (qleftright.c:45-46).
__device__ __forceinline__ Cons riemann_flux(const Phys& P, const Prim& ql, const Prim& qr) {
    const double gamma = P.gamma, smallr = P.smallr, smallc = P.smallc, smallp = P.smallp;
    const double gamma6 = P.gamma6;

    double rl = cfmax(ql.r, smallr);
    double ul = ql.u;
    double pl = cfmax(ql.p, rl * smallp);
    double rr = cfmax(qr.r, smallr);
    double ur = qr.u;
    double pr = cfmax(qr.p, rr * smallp);
    double cl = gamma * pl * rl;
    double cr = gamma * pr * rr;
    double wl = sqrt(cl);
    double wr = sqrt_eq(cr, cl, wl);  // equal states: cr == cl
    const double wl0 = wl, wr0 = wr;  // sqrt(cl), sqrt(cr)
    double pstar = cfmax(((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr), 0.0);

    for (int iter = 0; iter < P.niter; iter++) {
        double pst = pstar;
        double wwl = sqrt_eq(cl * (1.0 + zdiv(gamma6 * (pst - pl), pl)), cl, wl0);
        double wwr = sqrt_eq(cr * (1.0 + zdiv(gamma6 * (pst - pr), pr)), cr, wr0);
        double usl = ul - zdiv(pst - pl, wwl);
        double usr = ur + zdiv(pst - pr, wwr);
        const double dus = usl - usr;
        double tmp;
        if (dus == 0.0) {
            // q_r q_l / (q_r + q_l) is positive and finite (W_K > 0), so the
            // product with a signed zero is that zero: the step is dus itself,
            // without the three divisions.
            tmp = dus;
        } else {
            double swwl = wwl * wwl;
            double qlw = 2.0 * wwl * swwl / (swwl + cl);
            double qrw = 2.0 * wwr * (wwr * wwr) / ((wwr * wwr) + cr);
            tmp = (qrw * qlw / (qrw + qlw) * dus);
        }
        double delp = omax(tmp, (-pst));
        pst += delp;
        double tmp2 = zdiv(delp, pst + P.smallpp);
        double conv = fabs(tmp2);
        pstar = pst;
        if (!(conv > 1e-6)) break;
    }

    wr = sqrt_eq(cr * (1.0 + zdiv(gamma6 * (pstar - pr), pr)), cr, wr0);
    wl = sqrt_eq(cl * (1.0 + zdiv(gamma6 * (pstar - pl), pl)), cl, wl0);
    double ustar = 0.5 * (ul + zdiv(pl - pstar, wl) + ur - zdiv(pr - pstar, wr));
    bool left = ustar > 0.0;
    double sgnm = left ? 1.0 : -1.0;
    double ro = left ? rl : rr;
    double uo = left ? ul : ur;
    double po = left ? pl : pr;
    double wo = left ? wl : wr;
    const double co_raw = sqrt(fabs(gamma * po / ro));
    double co = cfmax(smallc, co_raw);
    double rstar = div1(ro, 1.0 + zdiv(ro * (po - pstar), wo * wo));
    rstar = cfmax(rstar, smallr);
    // With p* = p_o and rho* = rho_o (both positive: equal bits), c* repeats
    // c_o's arithmetic on the same operands.
    double cstar;
    if (pstar == po && rstar == ro) cstar = co_raw;
    else cstar = sqrt(fabs(gamma * pstar / rstar));
    cstar = cfmax(smallc, cstar);
    double spout = co - sgnm * uo;
    double spin = cstar - sgnm * ustar;
    double ushock = wo / ro - sgnm * uo;
    if (pstar >= po) {
        spin = ushock;
        spout = ushock;
    }
    double scr = cfmax(spout - spin, smallc + fabs(spout + spin));
    double frac = (1.0 + (spout + spin) / scr) * 0.5;
    frac = cfmax(0.0, cfmin(1.0, frac));
    double gr, gu, gp;
    if (spout < 0.0) {
        gr = ro;
        gu = uo;
        gp = po;
    } else if (spin > 0.0) {
        gr = rstar;
        gu = ustar;
        gp = pstar;
    } else {
        gr = (frac * rstar + (1.0 - frac) * ro);
        gu = (frac * ustar + (1.0 - frac) * uo);
        gp = (frac * pstar + (1.0 - frac) * po);
    }
    double gv = left ? ql.v : qr.v;

    Cons f;
    double mass = gr * gu;
    f.d = mass;
    f.mn = mass * gu + gp;
    f.mt = mass * gv;
    double ekin = 0.5 * gr * ((gu * gu) + (gv * gv));
    double etot = gp * P.entho + ekin;
    f.e = gu * (etot + gp);
    return f;
}

// conservar.c:166-172: u + (F_left - F_right) * dtdx, difference first.
__device__ __forceinline__ Cons update(const Cons& u, const Cons& fl, const Cons& fr, double dtdx) {
    Cons o;
    o.d = u.d + (fl.d - fr.d) * dtdx;
    o.mn = u.mn + (fl.mn - fr.mn) * dtdx;
    o.mt = u.mt + (fl.mt - fr.mt) * dtdx;
    o.e = u.e + (fl.e - fr.e) * dtdx;
    return o;
}

// Courant speeds of one updated cell: ComputeQEforRow.c:31-47,
// equation_of_state.c:41-48, courantOnXY.c:44-45.  cn / ct: c + |u| along the
// sweep's normal / transverse direction.
__device__ __forceinline__ void courant_speeds(const Phys& P, const Cons& u, double& cn,
                                               double& ct) {
    Prim q;
    double c;
    cons_to_prim(P, u, q, c);
    cn = c + fabs(q.u);
    ct = c + fabs(q.v);
}

// The exact FP64 stage set used by the plain sweep (hb_march.cuh).
template <bool UNIT>
struct ExactStages {
    using Consts = Phys;
    using Prim = hb::Prim;
    using Flux = Cons;
    using Real = double;   // element type of Prim
    using Sound = double;  // the sound speed, from prim to trace
    using TraceK = hb::TraceK;
    // Staging the y march's cells by cp.async (the mixed set's column ring)
    // measured slower for the FP64 sets (4096^2: 0.791 against 0.760 ms).
    static constexpr bool async_ring = false;
    static constexpr int ring_ahead = 1;      // rows the ring copies ahead
    static constexpr int cells_per_lane = 1;  // x sweep window (hb_march.cuh)
    static __device__ __forceinline__ Consts consts(const Phys& P) { return P; }
    static __device__ __forceinline__ Prim zero_prim() { return Prim{0.0, 0.0, 0.0, 0.0}; }
    static __device__ __forceinline__ Flux zero_flux() { return Flux{0.0, 0.0, 0.0, 0.0}; }
    static __device__ __forceinline__ Sound zero_sound() { return 0.0; }
    static __device__ __forceinline__ TraceK trace_constants(const Phys& P, double dtdx) {
        return hb::trace_constants(P.scheme, dtdx);
    }
    static __device__ __forceinline__ bool second_order(const Phys& P) { return P.iorder != 1; }
    static __device__ __forceinline__ void prim(const Phys& P, const Cons& u, Prim& q, double& c) {
        cons_to_prim(P, u, q, c);
    }
    static __device__ __forceinline__ void slope4(const Phys& P, const Prim& a, const Prim& b,
                                                  const Prim& c, Prim& dq) {
        hb::slope4<UNIT>(P.slope_type, a, b, c, dq);
    }
    static __device__ __forceinline__ void trace(const TraceK& K, const Prim& q, const Prim& dq,
                                                 double c, Prim& xm, Prim& xp) {
        trace1(K, q, dq, c, xm, xp);
    }
    static __device__ __forceinline__ Flux riemann(const Phys& P, const Prim& l, const Prim& r) {
        return riemann_flux(P, l, r);
    }
    static __device__ __forceinline__ Cons update(const Cons& u, const Flux& fl, const Flux& fr,
                                                  double dtdx) {
        return hb::update(u, fl, fr, dtdx);
    }
    static __device__ __forceinline__ void courant(const Phys& P, const Cons& u, double& cn,
                                                   double& ct) {
        courant_speeds(P, u, cn, ct);
    }
};

}  // namespace hb
