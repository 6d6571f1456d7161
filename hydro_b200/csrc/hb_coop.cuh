// hb_coop.cuh -- the cooperative line window shared by the sweep kernels.
//
// A CTA of G warps takes 32G consecutive cells [c - 2, c + 32G - 2) of one
// line (a row for the x sweep, a column for the y sweep), one cell per thread,
// and produces the updates of the N = 32G - 4 cells [c, c + N).  The stages
// exchange neighbours through shared memory instead of warp shuffles, so the
// window's halo costs 4 of 32G threads instead of 4 of every warp's 32 (the
// warp window of hb_march.cuh, line_window_1), and the Riemann problems, the
// dearest stage, are solved once per interface but for two:
//
//   phase 1  load cell k = c - 2 + t (fused make_boundary), primitives -> smem
//   phase 2  slope (neighbours from smem) + trace -> qxm (kept), qxp -> smem
//   phase 3  Riemann problem + flux at (k | k + 1) from qxm[k], qxp[k + 1] -> smem
//   phase 4  update of cell k with the fluxes of its two faces; store
//
// Every cell gets the same stage calls on the same inputs as in the marching
// and warp-window kernels, so the FP64 stage set gives the same bits.
#pragma once

#include "hb_march.cuh"

namespace hb {

// Shared memory of one window, structure of arrays (one 8- or 4-byte element
// per thread and variable: conflict-free accesses).
template <class S, int G>
struct CoopSmem {
    using Real = typename S::Real;
    static constexpr int T = 32 * G;
    Real q[4][T];    // primitives
    Real xp[4][T];   // qxp
    double f[4][T];  // flux at (k | k + 1)
};

template <class S, int G>
__device__ __forceinline__ void coop_put(typename S::Real (*dst)[32 * G], int t,
                                         const typename S::Prim& q) {
    dst[0][t] = q.r;
    dst[1][t] = q.u;
    dst[2][t] = q.v;
    dst[3][t] = q.p;
}

template <class S, int G>
__device__ __forceinline__ typename S::Prim coop_get(const typename S::Real (*src)[32 * G],
                                                     int t) {
    return typename S::Prim{src[0][t], src[1][t], src[2][t], src[3][t]};
}

// The outputs of window `win` of line `line` are [win * N, win * N + N) n
// [2, n - 2).  All threads of the CTA must call this (it has CTA barriers);
// `active` false makes a thread take part in the barriers only.  Warps whose
// cells all lie past the line's end skip the arithmetic.  Accumulates the
// fused Courant maxima of its outputs into cx, cy.
// `staged`: the window's interior cells are already in the stage (thread t's
// cell in staged[v][t], coop_stage_issue), else they are loaded here.
template <class S, int DIR, int G>
__device__ __forceinline__ void coop_window(const SweepArgs& a, const typename S::Consts& C,
                                            int line, int win, double dtdx, bool active,
                                            double& cx, double& cy, CoopSmem<S, G>& sm,
                                            const double (*staged)[32 * G] = nullptr) {
    using Prim = typename S::Prim;
    using Flux = typename S::Flux;
    constexpr int T = 32 * G, N = T - 4;
    const int t = threadIdx.x;
    const int c = win * N;                          // first output cell of the window
    const int k = c - 2 + t;                        // this thread's cell
    // Threads whose cell is past n + 1 feed nothing that is stored (the last
    // output cell n - 3 needs cells up to n - 1, traced from up to n): whole
    // warps of them skip the arithmetic of a short last window.
    const bool work = active && (c - 2 + (t & ~31)) <= a.n;
    const LineGeom<DIR> g(a, line);
    const typename S::TraceK K = S::trace_constants(C, dtdx);

    Cons u{1.0, 0.0, 0.0, 1.0};
    Prim q = S::zero_prim();
    typename S::Sound cs = S::zero_sound();
    if (work) {
        constexpr int mn = Slots<DIR>::mn, mt = Slots<DIR>::mt;
        if (staged && k >= 2 && k < a.n - 2)
            u = Cons{staged[0][t], staged[mn][t], staged[mt][t], staged[3][t]};
        else if (k >= 0 && k < a.n)
            u = load_cell<DIR>(a, g, k);
        S::prim(C, u, q, cs);
        coop_put<S, G>(sm.q, t, q);
    }
    __syncthreads();
    Prim xm = S::zero_prim();
    if (work) {
        const Prim qm = t > 0 ? coop_get<S, G>(sm.q, t - 1) : q;
        const Prim qp = t < T - 1 ? coop_get<S, G>(sm.q, t + 1) : q;
        Prim dq = S::zero_prim();
        if (S::second_order(C)) S::slope4(C, qm, q, qp, dq);
        Prim xp;
        S::trace(K, q, dq, cs, xm, xp);
        coop_put<S, G>(sm.xp, t, xp);
    }
    __syncthreads();
    Flux f = S::zero_flux();
    if (work) {
        const Prim xpn = t < T - 1 ? coop_get<S, G>(sm.xp, t + 1) : xm;
        f = S::riemann(C, xm, xpn);                 // interface (k | k + 1)
        sm.f[0][t] = f.d;
        sm.f[1][t] = f.mn;
        sm.f[2][t] = f.mt;
        sm.f[3][t] = f.e;
    }
    __syncthreads();
    if (work && t >= 2 && t < 2 + N && k >= 2 && k < a.n - 2) {
        const Flux fl{sm.f[0][t - 1], sm.f[1][t - 1], sm.f[2][t - 1], sm.f[3][t - 1]};
        const Cons o = S::update(u, fl, f, dtdx);
        store_cell<DIR>(a, g, k, o);
        if (a.courant) {
            double cn, ct;
            S::courant(C, o, cn, ct);
            if (DIR == 1) {
                cx = cx > cn ? cx : cn;
                cy = cy > ct ? cy : ct;
            } else {
                cx = cx > ct ? cx : ct;
                cy = cy > cn ? cy : cn;
            }
        }
    }
}

// Grid: x = lines, y = windows.  One window per CTA.
template <class S, int DIR, int G>
__device__ __forceinline__ void coop_body(const SweepArgs& a, const Phys& P) {
    __shared__ CoopSmem<S, G> sm;
    const int line = blockIdx.x;
    const int win = a.w_lo + (int)blockIdx.y;
    bool active = line < a.nlines && win < a.w_hi;
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;
    const typename S::Consts C = S::consts(P);
    coop_window<S, DIR, G>(a, C, line, win, dt / P.dx, active, cx, cy, sm);
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}

// Copies thread t's interior cell of window `win` into stage[v][t] with
// cp.async (one commit group; empty for a ghost or out-of-line cell).
template <int DIR, int G>
__device__ __forceinline__ void coop_stage_issue(const SweepArgs& a, const LineGeom<DIR>& g,
                                                 int win, double (*stage)[32 * G]) {
    constexpr int N = 32 * G - 4;
    const int t = threadIdx.x;
    const int k = win * N - 2 + t;
    if (k >= 2 && k < a.n - 2) {
        const double* p = a.in + g.at(k);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(&stage[v][t]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst),
                         "l"(p + v * a.vs)
                         : "memory");
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Grid: x = lines, y = runs of NW consecutive windows.  A CTA sweeps its run
// software-pipelined: while a window computes, each thread copies its cell of
// the next window into the other half of a shared-memory stage (its own slot
// only, so the copies need no barrier of their own).
template <class S, int DIR, int G, int NW>
__device__ __forceinline__ void coop_pipe_body(const SweepArgs& a, const Phys& P) {
    __shared__ CoopSmem<S, G> sm;
    __shared__ double stage[2][4][32 * G];
    const int line = blockIdx.x;
    const int total = (a.n - 2 + (32 * G - 4) - 1) / (32 * G - 4);
    const int w0 = a.w_lo + (int)blockIdx.y * NW;
    int w1 = w0 + NW;
    w1 = w1 < a.w_hi ? w1 : a.w_hi;
    w1 = w1 < total ? w1 : total;
    bool active = line < a.nlines && w0 < w1;   // uniform over the CTA
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;
    if (active) {
        const typename S::Consts C = S::consts(P);
        const LineGeom<DIR> g(a, line);
        coop_stage_issue<DIR, G>(a, g, w0, stage[0]);
        for (int w = w0; w < w1; w++) {
            const int b = (w - w0) & 1;
            if (w + 1 < w1) coop_stage_issue<DIR, G>(a, g, w + 1, stage[b ^ 1]);
            else asm volatile("cp.async.commit_group;\n" ::: "memory");
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            coop_window<S, DIR, G>(a, C, line, w, dt / P.dx, true, cx, cy, sm, stage[b]);
            __syncthreads();  // the window's shared memory is free for the next one
        }
    }
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}

// Windows per line of n cells (outputs [2, n - 2)).
template <int G>
__host__ __device__ constexpr int coop_windows(int n) {
    return (n - 2 + (32 * G - 4) - 1) / (32 * G - 4);
}

}  // namespace hb
