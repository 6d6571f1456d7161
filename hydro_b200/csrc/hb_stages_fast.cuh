// hb_stages_fast.cuh -- the FMA FP64 stage set of the sweep.
//
// The algorithm and the precision of the FP64 restatement (hb_stages.cuh,
// reference citations there), with the arithmetic freed from the reference's
// operation order:
//   * multiply-adds are contracted to FMA (this translation unit is built
//     with --fmad=true);
//   * divisions become multiplications by reciprocals, one reciprocal per
//     denominator (1/rho in constoprim and the Courant speeds; 1/c and 1/rho
//     in trace; 1/p_K, 1/W_K and 1/rho_o in the Riemann solver), and square
//     roots products with reciprocal square roots; reciprocals and reciprocal
//     square roots come from the hardware approximation refined by two
//     Newton-Raphson steps (hb_fastmath.cuh), to within about an ulp;
//   * the Newton iteration on p* carries W^2 and 1/W instead of W, and its
//     step is (u*_l - u*_r) / (1/q_l + 1/q_r), the reference's
//     q_l q_r / (q_l + q_r) (u*_l - u*_r) with one reciprocal (riemann.c:136-150).
// Each result differs from the reference's by a few ulps per operation; the
// state stays within 1e-12 (relative, per cell) of the reference's over the
// 200-step 4096^2 centred-blast run (tests/test_gpu_fast.py).  It is not
// bitwise: the Newton stopping test |dp / p| <= 1e-6 may take one iteration
// more or fewer than the reference's where the ratio lies within rounding of
// the threshold, and min/max selections in the limiters may go the other way
// on near-ties.
#pragma once

#include "hb_fastmath.cuh"
#include "hb_stages.cuh"

namespace hb {

// sqrt(x) for x >= 0 as x / sqrt(x) (0 for x = 0; the approximation of
// rsqrt(0) is infinite).
__device__ __forceinline__ double sqrt64(double x) { return x > 0.0 ? x * rsqrt64(x) : 0.0; }

struct FastConsts {
    Phys P;
    double inv_slope;  // 1 / slope_type
};

struct FastStages {
    using Consts = FastConsts;
    using Prim = hb::Prim;
    using Flux = Cons;
    using Real = double;   // element type of Prim
    using Sound = double;  // the sound speed, from prim to trace
    using TraceK = hb::TraceK;
    // Staging the y march's cells by cp.async (the mixed set's column ring)
    // measured slower for the FP64 sets (4096^2: 0.791 against 0.760 ms).
    static constexpr bool async_ring = false;
    static constexpr int ring_ahead = 1;      // rows the ring copies ahead
    static constexpr int cells_per_lane = 1;

    static __device__ __forceinline__ Consts consts(const Phys& P) {
        FastConsts C;
        C.P = P;
        C.inv_slope = 1.0 / P.slope_type;
        return C;
    }
    static __device__ __forceinline__ Prim zero_prim() { return Prim{0.0, 0.0, 0.0, 0.0}; }
    static __device__ __forceinline__ Flux zero_flux() { return Flux{0.0, 0.0, 0.0, 0.0}; }
    static __device__ __forceinline__ Sound zero_sound() { return 0.0; }
    static __device__ __forceinline__ TraceK trace_constants(const Consts& C, double dtdx) {
        return hb::trace_constants(C.P.scheme, dtdx);
    }
    static __device__ __forceinline__ bool second_order(const Consts& C) {
        return C.P.iorder != 1;
    }

    // constoprim.c:37-52, equation_of_state.c:41-48.
    static __device__ __forceinline__ void prim(const Consts& C, const Cons& u, Prim& q,
                                                double& c) {
        const Phys& P = C.P;
        const double r = fmax(u.d, P.smallr);
        const double ir = rcp64(r);
        const double un = u.mn * ir;
        const double ut = u.mt * ir;
        const double e = u.e * ir - 0.5 * (un * un + ut * ut);
        const double p = fmax(P.gm1 * r * e, r * P.smallp);
        q = Prim{r, un, ut, p};
        c = sqrt64(P.gamma * p * ir);
    }

    // slope.c:37-50.
    static __device__ __forceinline__ double slope1(const Consts& C, double qm, double q0,
                                                    double qp) {
        double dlft, drgt, dcen;
        if (C.P.unit_slope) {
            dlft = q0 - qm;
            drgt = qp - q0;
            dcen = 0.5 * (dlft + drgt);
        } else {
            dlft = C.P.slope_type * (q0 - qm);
            drgt = C.P.slope_type * (qp - q0);
            dcen = 0.5 * (dlft + drgt) * C.inv_slope;
        }
        const bool llftrgt = (dlft * drgt) <= 0.0;
        const double m = llftrgt ? 0.0 : fmin(fmin(fabs(dlft), fabs(drgt)), fabs(dcen));
        return (dcen > 0.0) ? m : -m;
    }
    static __device__ __forceinline__ void slope4(const Consts& C, const Prim& a, const Prim& b,
                                                  const Prim& c, Prim& dq) {
        if (hb::flat3(a, b, c)) {  // flat: every slope is -0, as slope1 computes
            dq = Prim{-0.0, -0.0, -0.0, -0.0};
            return;
        }
        dq.r = slope1(C, a.r, b.r, c.r);
        dq.u = slope1(C, a.u, b.u, c.u);
        dq.v = slope1(C, a.v, b.v, c.v);
        dq.p = slope1(C, a.p, b.p, c.p);
    }

    // trace.c:63-123.
    static __device__ __forceinline__ void trace(const TraceK& K, const Prim& q, const Prim& dq,
                                                 double cc, Prim& qxm, Prim& qxp) {
        if (dq.r == 0.0 && dq.u == 0.0 && dq.v == 0.0 && dq.p == 0.0) {
            // A flat cell: every characteristic amplitude is zero, so both
            // traced states are the cell's own (the general form can only
            // differ in the sign of a zero velocity).
            qxp = q;
            qxm = q;
            return;
        }
        const double dtdx = K.dtdx;
        const double csq = cc * cc;
        const double icc = rcp64(cc);
        const double ir = rcp64(q.r);
        const double rOcc = q.r * icc;
        const double OrOcc = cc * ir;
        const double dprcc = dq.p * ir * icc;
        const double alpham = 0.5 * (dprcc - dq.u) * rOcc;
        const double alphap = 0.5 * (dprcc + dq.u) * rOcc;
        const double alpha0r = dq.r - dq.p * (icc * icc);
        const double alpha0v = dq.v;
        const double upcc = q.u + cc, umcc = q.u - cc;
        const double upccx = upcc * dtdx, umccx = umcc * dtdx, ux = q.u * dtdx;

        double spm = (umcc >= K.zeror) ? K.project : umccx + 1.0;
        double spp = (upcc >= K.zeror) ? K.project : upccx + 1.0;
        double spz = (q.u >= K.zeror) ? K.project : ux + 1.0;
        double ap = -0.5 * spp * alphap, am = -0.5 * spm * alpham;
        double azr = -0.5 * spz * alpha0r, azv = -0.5 * spz * alpha0v;
        qxp = Prim{q.r + (ap + am + azr), q.u + (ap - am) * OrOcc, q.v + azv,
                   q.p + (ap + am) * csq};

        spm = (umcc <= K.zerol) ? -K.project : umccx - 1.0;
        spp = (upcc <= K.zerol) ? -K.project : upccx - 1.0;
        spz = (q.u <= K.zerol) ? -K.project : ux - 1.0;
        ap = -0.5 * spp * alphap;
        am = -0.5 * spm * alpham;
        azr = -0.5 * spz * alpha0r;
        azv = -0.5 * spz * alpha0v;
        qxm = Prim{q.r + (ap + am + azr), q.u + (ap - am) * OrOcc, q.v + azv,
                   q.p + (ap + am) * csq};
    }

    // riemann.c:89-258 and cmpflx.c:52-73, with the C99 selection order.
    static __device__ __forceinline__ Flux riemann(const Consts& C, const Prim& ql,
                                                   const Prim& qr) {
        const Phys& P = C.P;
        const double rl = fmax(ql.r, P.smallr), ul = ql.u;
        const double pl = fmax(ql.p, rl * P.smallp);
        const double rr = fmax(qr.r, P.smallr), ur = qr.u;
        const double pr = fmax(qr.p, rr * P.smallp);
        double gr, gu, gp, gv;  // the state sampled at the interface
        if (pl == pr && ul == ur) {
            // Equal pressure and velocity on both sides (at rest, a uniform
            // flow or a pure contact): the exact solution p* = p, u* = u, where
            // the reference's iteration lands within rounding of p; the
            // interface samples the upwind side's state (the right for u = 0).
            const bool left = ul > 0.0;
            gr = left ? rl : rr;
            gu = ul;
            gp = pl;
            gv = left ? ql.v : qr.v;
        } else {
            const double cl = P.gamma * pl * rl;
            const double cr = P.gamma * pr * rr;
            // W_K^2 = c_K (1 + gamma6 (p - p_K) / p_K) = c_K + k_K (p - p_K).
            const double kl = cl * P.gamma6 * rcp64(pl);
            const double kr = cr * P.gamma6 * rcp64(pr);
            const double il0 = rsqrt64(cl), ir0 = rsqrt64(cr);  // 1 / W at p = p_K
            double il = il0, ir = ir0;
            const double wl0 = cl * il, wr0 = cr * ir;
            double pst =
                fmax(((wr0 * pl + wl0 * pr) + wl0 * wr0 * (ul - ur)) * rcp64(wl0 + wr0), 0.0);

            // Where p equals p_K, W^2 is c_K and 1/W is known (the usual case
            // between equal states); a zero velocity jump makes the step zero.
            for (int iter = 0; iter < P.niter; iter++) {
                const double wl2 = fma(kl, pst - pl, cl);
                const double wr2 = fma(kr, pst - pr, cr);
                il = il0;
                if (wl2 != cl) il = rsqrt64(wl2);
                ir = ir0;
                if (wr2 != cr) ir = rsqrt64(wr2);
                const double usl = ul - (pst - pl) * il;
                const double usr = ur + (pst - pr) * ir;
                const double dus = usl - usr;
                double delp = 0.0;
                if (dus != 0.0) {
                    // 1/q_K = (W^2 + c_K) / (2 W^3)
                    const double iql = 0.5 * (wl2 + cl) * (il * il * il);
                    const double iqr = 0.5 * (wr2 + cr) * (ir * ir * ir);
                    delp = dus * rcp64(iql + iqr);
                }
                delp = delp > -pst ? delp : -pst;
                pst += delp;
                if (!(fabs(delp) > 1e-6 * (pst + P.smallpp))) break;
            }
            const double pstar = pst;

            const double wr2 = fma(kr, pstar - pr, cr);
            const double wl2 = fma(kl, pstar - pl, cl);
            ir = ir0;
            if (wr2 != cr) ir = rsqrt64(wr2);
            il = il0;
            if (wl2 != cl) il = rsqrt64(wl2);
            const double ustar = 0.5 * (ul + (pl - pstar) * il + ur - (pr - pstar) * ir);
            const bool left = ustar > 0.0;
            const double sgnm = left ? 1.0 : -1.0;
            const double ro = left ? rl : rr;
            const double uo = left ? ul : ur;
            const double po = left ? pl : pr;
            const double wo2 = left ? wl2 : wr2;
            const double wo = wo2 * (left ? il : ir);
            const double iro = rcp64(ro);
            const double co = fmax(P.smallc, sqrt64(fabs(P.gamma * po * iro)));
            double rstar = ro * rcp64(1.0 + ro * (po - pstar) * rcp64(wo2));
            rstar = fmax(rstar, P.smallr);
            const double cstar = fmax(P.smallc, sqrt64(fabs(P.gamma * pstar * rcp64(rstar))));
            double spout = co - sgnm * uo;
            double spin = cstar - sgnm * ustar;
            const double ushock = wo * iro - sgnm * uo;
            if (pstar >= po) {
                spin = ushock;
                spout = ushock;
            }
            const double scr = fmax(spout - spin, P.smallc + fabs(spout + spin));
            const double frac = fmax(0.0, fmin(1.0, (1.0 + (spout + spin) * rcp64(scr)) * 0.5));
            if (spout < 0.0) {
                gr = ro;
                gu = uo;
                gp = po;
            } else if (spin > 0.0) {
                gr = rstar;
                gu = ustar;
                gp = pstar;
            } else {
                gr = frac * rstar + (1.0 - frac) * ro;
                gu = frac * ustar + (1.0 - frac) * uo;
                gp = frac * pstar + (1.0 - frac) * po;
            }
            gv = left ? ql.v : qr.v;
        }
        Cons f;
        const double mass = gr * gu;
        f.d = mass;
        f.mn = mass * gu + gp;
        f.mt = mass * gv;
        const double ekin = 0.5 * gr * (gu * gu + gv * gv);
        const double etot = gp * P.entho + ekin;
        f.e = gu * (etot + gp);
        return f;
    }

    // conservar.c:166-172.
    static __device__ __forceinline__ Cons update(const Cons& u, const Flux& fl, const Flux& fr,
                                                  double dtdx) {
        return Cons{fma(fl.d - fr.d, dtdx, u.d), fma(fl.mn - fr.mn, dtdx, u.mn),
                    fma(fl.mt - fr.mt, dtdx, u.mt), fma(fl.e - fr.e, dtdx, u.e)};
    }

    // ComputeQEforRow.c:31-47, equation_of_state.c:41-48, courantOnXY.c:44-45.
    static __device__ __forceinline__ void courant(const Consts& C, const Cons& u, double& cn,
                                                   double& ct) {
        Prim q;
        double c;
        prim(C, u, q, c);
        cn = c + fabs(q.u);
        ct = c + fabs(q.v);
    }
};

}  // namespace hb
