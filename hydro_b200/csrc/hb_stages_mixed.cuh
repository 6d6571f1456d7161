// hb_stages_mixed.cuh -- the mixed-precision stage set of the sweep.
//
// Same algorithm as the FP64 restatement (hb_stages.cuh, reference citations
// there), with the precision split:
//   FP32: constoprim, equation_of_state, slope, trace, the Riemann first guess
//         and state sampling, cmpflx;
//   FP64: the Newton iteration on the star pressure (riemann.c:126-156), the
//         conservative update u + dt/dx (F_l - F_r) with the flux difference
//         taken in FP64 from the FP32 fluxes, and the Courant speeds that feed
//         the dt reduction.
// The state in HBM stays FP64.  It is not bitwise comparable to the reference
// and is validated by its L1 / Linf error against the FP64 path.
//
// Every multiply-add that should fuse is written as fmaf / fma, and the
// translation unit is built without FMA contraction (--fmad=false, with fast
// FP32 division and square root): the compiler then fuses nothing on its own,
// so each stage rounds the same way in every kernel that calls it, whatever
// its register budget, thread count or surroundings.  A batched instance is
// therefore bitwise equal to its single-grid run under any kernel, tiling or
// launch shape.
#pragma once

#include "hb_kernels.cuh"
#include "hb_fastmath.cuh"

namespace hb {

struct PrimF {
    float r, u, v, p;
};

struct FluxF {
    float d, mn, mt, e;
};

struct MixedConsts {
    float gamma, gm1, smallr, smallc, smallp, gamma6, entho, slope_type;
    float inv_slope;                          // 1 / slope_type (slope.c:44 divides)
    int unit_slope;                           // slope_type == 1
    double gamma6d, smallppd;                 // Newton iteration
    double gammad, gm1d, smallrd, smallpd;    // Courant speeds
    int niter, iorder, scheme;
};

// What the primitives step hands to the trace step: the sound speed c with
// 1/c and 1/rho, which the trace needs and prim has on hand (one reciprocal
// square root gives c and 1/c).
struct SoundF {
    float c, ic, ir;
};

struct TraceKF {
    float dtdx, zerol, zeror, project;
};

struct MixedStages {
    using Consts = MixedConsts;
    using Prim = PrimF;
    using Flux = Cons;   // the FP32 flux converted once to FP64 (exact)
    using Real = float;     // element type of Prim
    using Sound = SoundF;
    using TraceK = TraceKF;
    // The y march stages its cells with cp.async into a shared-memory ring,
    // three rows ahead (4096^2 y sweep: 0.208 ms, against 0.212 ms two rows
    // ahead, 0.235 ms one row ahead and 0.355 ms prefetching one row into
    // registers).
    static constexpr bool async_ring = true;
    static constexpr int ring_ahead = 3;      // rows the ring copies ahead
    static constexpr int cells_per_lane = 2;  // x sweep window (hb_march.cuh)

    static __device__ __forceinline__ Consts consts(const Phys& P) {
        Consts C;
        C.gamma = (float)P.gamma;
        C.gm1 = (float)P.gm1;
        C.smallr = (float)P.smallr;
        C.smallc = (float)P.smallc;
        C.smallp = (float)P.smallp;
        C.gamma6 = (float)P.gamma6;
        C.entho = (float)P.entho;
        C.slope_type = (float)P.slope_type;
        C.inv_slope = (float)(1.0 / P.slope_type);
        C.unit_slope = P.unit_slope;
        C.gamma6d = P.gamma6;
        C.smallppd = P.smallpp;
        C.gammad = P.gamma;
        C.gm1d = P.gm1;
        C.smallrd = P.smallr;
        C.smallpd = P.smallp;
        C.niter = P.niter;
        C.iorder = P.iorder;
        C.scheme = P.scheme;
        return C;
    }
    static __device__ __forceinline__ Prim zero_prim() { return Prim{0.f, 0.f, 0.f, 0.f}; }
    static __device__ __forceinline__ Flux zero_flux() { return Flux{0.0, 0.0, 0.0, 0.0}; }
    static __device__ __forceinline__ Sound zero_sound() { return Sound{0.f, 0.f, 0.f}; }
    static __device__ __forceinline__ bool second_order(const Consts& C) { return C.iorder != 1; }

    static __device__ __forceinline__ TraceK trace_constants(const Consts& C, double dtdx) {
        TraceK k;
        k.dtdx = (float)dtdx;
        k.zerol = 0.f;
        k.zeror = 0.f;
        k.project = 0.f;
        if (C.scheme == 1) {
            k.zerol = (float)(-100.0 / dtdx);
            k.zeror = (float)(100.0 / dtdx);
            k.project = 1.f;
        }
        if (C.scheme == 2) k.project = 1.f;
        return k;
    }

    static __device__ __forceinline__ void prim(const Consts& C, const Cons& u, Prim& q, Sound& c) {
        const float r = fmaxf((float)u.d, C.smallr);
        const float ir = 1.0f / r;
        const float un = (float)u.mn * ir;
        const float ut = (float)u.mt * ir;
        const float eken = 0.5f * fmaf(un, un, ut * ut);
        const float e = fmaf((float)u.e, ir, -eken);
        const float p = fmaxf(C.gm1 * r * e, r * C.smallp);
        q = Prim{r, un, ut, p};
        const float c2 = C.gamma * p * ir;
        const float ic = rsqrtf(c2);
        c = Sound{c2 * ic, ic, ir};
    }

    // slope.c:37-50; with slope_type 1 the two scalings are skipped.
    static __device__ __forceinline__ float slope1(const Consts& C, float qm, float q0, float qp) {
        float dlft = q0 - qm, drgt = qp - q0, dcen;
        if (C.unit_slope) {
            dcen = 0.5f * (dlft + drgt);
        } else {
            dlft *= C.slope_type;
            drgt *= C.slope_type;
            dcen = 0.5f * (dlft + drgt) * C.inv_slope;
        }
        const float lim = (dlft * drgt <= 0.f) ? 0.f : fminf(fabsf(dlft), fabsf(drgt));
        const float m = fminf(lim, fabsf(dcen));
        return dcen > 0.f ? m : -m;
    }
    static __device__ __forceinline__ void slope4(const Consts& C, const Prim& a, const Prim& b,
                                                  const Prim& c, Prim& dq) {
        // A flat neighbourhood (every difference exactly zero, so no
        // infinities) gives -0 for every slope, as slope1 computes.
        if (b.r - a.r == 0.f && c.r - b.r == 0.f && b.u - a.u == 0.f && c.u - b.u == 0.f &&
            b.v - a.v == 0.f && c.v - b.v == 0.f && b.p - a.p == 0.f && c.p - b.p == 0.f) {
            dq = Prim{-0.f, -0.f, -0.f, -0.f};
            return;
        }
        dq.r = slope1(C, a.r, b.r, c.r);
        dq.u = slope1(C, a.u, b.u, c.u);
        dq.v = slope1(C, a.v, b.v, c.v);
        dq.p = slope1(C, a.p, b.p, c.p);
    }

    // trace.c:63-123, with the factor -1/2 of the characteristic amplitudes
    // folded into them once for both sides.
    static __device__ __forceinline__ void trace(const TraceK& K, const Prim& q, const Prim& dq,
                                                 const Sound& s, Prim& qxm, Prim& qxp) {
        if (dq.r == 0.f && dq.u == 0.f && dq.v == 0.f && dq.p == 0.f) {
            // A flat cell: every characteristic amplitude below is zero, so
            // both traced states are the cell's own (the general form can only
            // differ in the sign of a zero velocity).
            qxp = q;
            qxm = q;
            return;
        }
        const float cc = s.c, icc = s.ic, ir = s.ir;
        const float csq = cc * cc;
        const float rOcc = q.r * icc;
        const float OrOcc = cc * ir;
        const float dprcc = dq.p * ir * icc;
        const float hm = -0.25f * rOcc;                       // -1/2 * 1/2 rho/c
        const float am0 = (dprcc - dq.u) * hm;                 // -alpham / 2
        const float ap0 = (dprcc + dq.u) * hm;                 // -alphap / 2
        const float azr0 = -0.5f * fmaf(-dq.p, icc * icc, dq.r);  // -alpha0r / 2
        const float azv0 = -0.5f * dq.v;                       // -alpha0v / 2
        const float upcc = q.u + cc, umcc = q.u - cc;

        float spm = (umcc >= K.zeror) ? K.project : fmaf(umcc, K.dtdx, 1.f);
        float spp = (upcc >= K.zeror) ? K.project : fmaf(upcc, K.dtdx, 1.f);
        float spz = (q.u >= K.zeror) ? K.project : fmaf(q.u, K.dtdx, 1.f);
        float ap = spp * ap0, am = spm * am0, azr = spz * azr0, azv = spz * azv0;
        qxp = Prim{q.r + (ap + am + azr), fmaf(ap - am, OrOcc, q.u), q.v + azv,
                   fmaf(ap + am, csq, q.p)};

        spm = (umcc <= K.zerol) ? -K.project : fmaf(umcc, K.dtdx, -1.f);
        spp = (upcc <= K.zerol) ? -K.project : fmaf(upcc, K.dtdx, -1.f);
        spz = (q.u <= K.zerol) ? -K.project : fmaf(q.u, K.dtdx, -1.f);
        ap = spp * ap0;
        am = spm * am0;
        azr = spz * azr0;
        azv = spz * azv0;
        qxm = Prim{q.r + (ap + am + azr), fmaf(ap - am, OrOcc, q.u), q.v + azv,
                   fmaf(ap + am, csq, q.p)};
    }

    static __device__ __forceinline__ Flux riemann(const Consts& C, const Prim& ql, const Prim& qr) {
        // First guess (FP32).
        float rl = fmaxf(ql.r, C.smallr), pl = fmaxf(ql.p, rl * C.smallp);
        float rr = fmaxf(qr.r, C.smallr), pr = fmaxf(qr.p, rr * C.smallp);
        const float ul = ql.u, ur = qr.u;
        float cl = C.gamma * pl * rl, cr = C.gamma * pr * rr;
        // gamma p rho multiplies two small numbers: near vacuum (density near
        // smallr, pressure near smallp) it falls below the FP32 normal range
        // and would be flushed to zero.  The solve is covariant under scaling
        // density and pressure by one factor a (velocities and sound speeds
        // unchanged; rho*, p*, W and the fluxes scale by a, W^2 by a^2), so
        // such an interface is solved with both scaled by a = 2^k, which is
        // exact, and its flux scaled back in FP64.  Other interfaces have
        // k = 0 and the arithmetic is untouched.
        float a = 1.f;
        if (!(cl >= 1e-30f && cr >= 1e-30f)) {
            const int e = ilogbf(rl) + ilogbf(pl) + ilogbf(rr) + ilogbf(pr);
            a = ldexpf(1.f, -e / 4);  // geometric mean of rho p on both sides near 1
            rl *= a; pl *= a; rr *= a; pr *= a;
            cl = C.gamma * pl * rl;
            cr = C.gamma * pr * rr;
        }
        float gr, gu, gp, gv;  // the state sampled at the interface
        if (pl == pr && ul == ur) {
            // Equal pressure and velocity on both sides (a state at rest, a
            // uniform flow or a pure contact): the exact solution is p* = p and
            // u* = u, at which every Newton step is exactly zero, and the
            // interface samples the upwind side's state (right for u = 0),
            // whichever of the sampling's branches applies.
            const bool left = ul > 0.f;
            gr = left ? rl : rr;
            gu = ul;
            gp = pl;
            gv = left ? ql.v : qr.v;
        } else {
            const float wl0 = sqrtf(cl), wr0 = sqrtf(cr);
            const float p0 =
                fmaxf(fmaf(wl0 * wr0, ul - ur, fmaf(wr0, pl, wl0 * pr)) / (wl0 + wr0), 0.f);

            // Newton iteration on p* (FP64): W^2 = c (1 + gamma6 (p - p_K) / p_K),
            // u*_l = u_l - (p - p_l) / W_l, u*_r = u_r + (p - p_r) / W_r, step
            // dp = (q_l q_r / (q_l + q_r)) (u*_l - u*_r) with q = 2 W^3 / (W^2 + c).
            const double pld = pl, prd = pr, cld = cl, crd = cr, uld = ul, urd = ur;
            const double kl = cld * C.gamma6d * rcp64(pld);
            const double kr = crd * C.gamma6d * rcp64(prd);
            double pst = p0;
            for (int iter = 0; iter < C.niter; iter++) {
                const double wl2d = fma(kl, pst - pld, cld);
                const double wr2d = fma(kr, pst - prd, crd);
                const double il = rsqrt64(wl2d), ir = rsqrt64(wr2d);
                const double usl = fma(-(pst - pld), il, uld);
                const double usr = fma(pst - prd, ir, urd);
                const double iql = 0.5 * (wl2d + cld) * (il * il * il);
                const double iqr = 0.5 * (wr2d + crd) * (ir * ir * ir);  // 1/q = (W^2+c)/(2W^3)
                double delp = (usl - usr) * rcp64(iql + iqr);
                delp = delp > -pst ? delp : -pst;
                pst += delp;
                if (!(fabs(delp) > 1e-6 * fabs(pst + C.smallppd * a))) break;
            }
            const float ps = (float)pst;

            // Sampling (FP32).  W^2 at p* from the iteration's coefficients, and
            // 1/W by one reciprocal square root per side (W = W^2 / W).
            const float wl2 = (float)fma(kl, pst - pld, cld);
            const float wr2 = (float)fma(kr, pst - prd, crd);
            const float iwl = rsqrtf(wl2), iwr = rsqrtf(wr2);
            const float wl = wl2 * iwl, wr = wr2 * iwr;
            // u* grouped as (ul + ur) + (left term - right term): a mirror pair
            // (a reflecting wall: ur = -ul, identical pressures and W) gives
            // u* = 0 exactly, so the wall's mass and energy fluxes vanish
            // exactly.  The reference's order, ul + A_l + ur - A_r, leaves FP32
            // rounding of A, which is large next to near-vacuum states.
            const float ustar = 0.5f * ((ul + ur) + ((pl - ps) * iwl - (pr - ps) * iwr));
            const bool left = ustar > 0.f;
            const float sgnm = left ? 1.f : -1.f;
            const float ro = left ? rl : rr, uo = left ? ul : ur, po = left ? pl : pr;
            const float wo = left ? wl : wr;
            const float iwo = left ? iwl : iwr;
            const float iro = 1.0f / ro;
            const float co = fmaxf(C.smallc, sqrtf(fabsf(C.gamma * po * iro)));
            const float den = fmaf(ro * (po - ps), iwo * iwo, 1.f);
            const float rstar_raw = ro / den;
            const float rstar = fmaxf(rstar_raw, C.smallr * a);
            float irs = den * iro;  // 1 / rho* = den / rho_o, unless the floor applies
            if (rstar != rstar_raw) irs = 1.0f / rstar;
            const float cstar = fmaxf(C.smallc, sqrtf(fabsf(C.gamma * ps * irs)));
            float spout = fmaf(-sgnm, uo, co);
            float spin = fmaf(-sgnm, ustar, cstar);
            const float ushock = fmaf(wo, iro, -sgnm * uo);
            if (ps >= po) {
                spin = ushock;
                spout = ushock;
            }
            const float scr = fmaxf(spout - spin, C.smallc + fabsf(spout + spin));
            const float frac = fmaxf(0.f, fminf(1.f, fmaf((spout + spin) / scr, 0.5f, 0.5f)));
            if (spout < 0.f) {
                gr = ro;
                gu = uo;
                gp = po;
            } else if (spin > 0.f) {
                gr = rstar;
                gu = ustar;
                gp = ps;
            } else {
                gr = fmaf(frac, rstar, (1.f - frac) * ro);
                gu = fmaf(frac, ustar, (1.f - frac) * uo);
                gp = fmaf(frac, ps, (1.f - frac) * po);
            }
            gv = left ? ql.v : qr.v;
        }
        const float mass = gr * gu;
        const float ekin = 0.5f * gr * fmaf(gu, gu, gv * gv);
        const float etot = fmaf(gp, C.entho, ekin);
        const FluxF f{mass, fmaf(mass, gu, gp), mass * gv, gu * (etot + gp)};
        Flux out{(double)f.d, (double)f.mn, (double)f.mt, (double)f.e};
        if (a != 1.f) {
            const double ia = 1.0 / (double)a;  // a power of two: exact
            out.d *= ia;
            out.mn *= ia;
            out.mt *= ia;
            out.e *= ia;
        }
        return out;
    }

    // FP64 update with the flux difference formed in FP64 (the FP32 fluxes
    // are exact in FP64, so no digits are lost to cancellation).
    static __device__ __forceinline__ Cons update(const Cons& u, const Flux& fl, const Flux& fr,
                                                  double dtdx) {
        return Cons{fma(fl.d - fr.d, dtdx, u.d), fma(fl.mn - fr.mn, dtdx, u.mn),
                    fma(fl.mt - fr.mt, dtdx, u.mt), fma(fl.e - fr.e, dtdx, u.e)};
    }

    // Courant speeds of the updated cell in FP64 (ComputeQEforRow +
    // equation_of_state + courantOnXY).
    static __device__ __forceinline__ void courant(const Consts& C, const Cons& u, double& cn,
                                                   double& ct) {
        const double r = u.d > C.smallrd ? u.d : C.smallrd;
        const double ir = rcp64(r);
        const double un = u.mn * ir, ut = u.mt * ir;
        const double e = fma(u.e, ir, -0.5 * fma(un, un, ut * ut));
        double p = C.gm1d * r * e;
        p = p > r * C.smallpd ? p : r * C.smallpd;
        const double c2 = C.gammad * p * ir;
        const double c = c2 * rsqrt64(c2);
        cn = c + fabs(un);
        ct = c + fabs(ut);
    }
};

}  // namespace hb
