// hb_march.cuh -- the line-marching skeleton shared by the sweep kernels.
//
// One thread owns a segment [k0, k1) of one line (a row for the x sweep, a
// column for the y sweep) and marches along it with a five-cell window:
//
//   iteration k: load cell k (fused make_boundary for ghost cells), its
//                primitives; slope + trace of cell k-1; Riemann problem + flux
//                at the interface (k-2 | k-1); update of cell k-2 with the
//                fluxes on its two faces; store.
//
// The arithmetic of each stage comes from a stage set S (hb_stages.cuh: the
// FP64 restatement of the reference; hb_stages_mixed.cuh: the mixed-precision
// form).  The state is always FP64 in HBM: 4 doubles read and 4 written per
// cell and sweep, plus a 4-cell halo per segment.
#pragma once

#include "hb_kernels.cuh"

namespace hb {

template <int DIR>
struct LineGeom {
    // DIR 1: line = row j = l + 2, cells along x.  DIR 2: line = column i = l + 2.
    long long base;   // offset of cell k = 0 of the line, variable 0
    long long step;   // offset between consecutive cells of the line
    __device__ __forceinline__ LineGeom(const SweepArgs& a, int l) {
        if (DIR == 1) {
            base = (long long)a.nxt * (l + 2);
            step = 1;
        } else {
            base = l + 2;
            step = a.nxt;
        }
    }
    __device__ __forceinline__ long long at(int k) const { return base + step * k; }
};

// Slots of the normal and transverse momentum: IU/IV for x, IV/IU for y
// (the swap of conservar.c:97-100 and :215-222).
template <int DIR> struct Slots;
template <> struct Slots<1> { static constexpr int mn = 1, mt = 2; };
template <> struct Slots<2> { static constexpr int mn = 2, mt = 1; };

// Ghost source of make_boundary.c:53-198 for position k of a line of n cells
// (nl = n - 4 interior cells).  Returns -1 when the side has no boundary fill.
template <int DIR>
__device__ __forceinline__ int ghost_source(int bt, int k, int n) {
    const int nl = n - 4;
    if (bt <= 0) return -1;
    if (k < 2) {
        if (bt == 1) return 3 - k;                 // reflect
        if (bt == 2) return DIR == 1 ? 2 : 4;      // "absorb" (x: col 2, y: row 4)
        return nl + k;                             // periodic
    }
    if (bt == 1) return 2 * nl + 3 - k;
    if (bt == 2) return DIR == 1 ? nl + 2 : nl + 1;
    return k - nl;
}

template <int DIR>
__device__ __forceinline__ Cons load_interior(const SweepArgs& a, const LineGeom<DIR>& g, int k) {
    constexpr int mn = Slots<DIR>::mn, mt = Slots<DIR>::mt;
    const double* __restrict__ p = a.in + g.at(k);
    return Cons{__ldg(p), __ldg(p + mn * a.vs), __ldg(p + mt * a.vs), __ldg(p + 3 * a.vs)};
}

template <int DIR>
__device__ __forceinline__ Cons load_cell(const SweepArgs& a, const LineGeom<DIR>& g, int k) {
    constexpr int mn = Slots<DIR>::mn, mt = Slots<DIR>::mt;
    const long long vs = a.vs;
    if (k >= 2 && k < a.n - 2) return load_interior<DIR>(a, g, k);
    // Ghost cell: the fused make_boundary.
    const int bt = (k < 2) ? a.bnd_lo : a.bnd_hi;
    const int src = ghost_source<DIR>(bt, k, a.n);
    double v[4];
    if (src < 0) {
        const double* p = a.resid + g.at(k);
        for (int s = 0; s < 4; s++) v[s] = p[s * vs];
    } else {
        const bool interior = src >= 2 && src < a.n - 2;
        const double* p = (interior ? a.in : a.resid) + g.at(src);
        const double sn = (bt == 1) ? -1.0 : 1.0;  // reflect flips the normal momentum
        for (int s = 0; s < 4; s++) v[s] = p[s * vs] * (s == mn ? sn : 1.0);
        if (a.gout) {
            double* q = a.gout + g.at(k);
            for (int s = 0; s < 4; s++) q[s * vs] = v[s];
        }
    }
    return Cons{v[0], v[mn], v[mt], v[3]};
}

template <int DIR>
__device__ __forceinline__ void store_cell(const SweepArgs& a, const LineGeom<DIR>& g, int k,
                                           const Cons& o) {
    constexpr int mn = Slots<DIR>::mn, mt = Slots<DIR>::mt;
    double* p = a.out + g.at(k);
    p[0] = o.d;
    p[mn * a.vs] = o.mn;
    p[mt * a.vs] = o.mt;
    p[3 * a.vs] = o.e;
}

// Slot of this CTA in a Courant accumulator array (see kCourSlots).
__device__ __forceinline__ int cour_slot() {
    return (int)((blockIdx.x + (unsigned long long)blockIdx.y * gridDim.x) % kCourSlots);
}

__device__ __forceinline__ void warp_max_atomic(unsigned long long* dst, double v) {
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = v > w ? v : w;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// Row staging of the x sweep.  A thread walking its own row would fetch each
// 32-byte sector four times (once per cell) from a thrashed L1; instead it
// fetches the four cells of a sector at once (two 16-byte loads per variable
// when the row is 16-byte aligned) into its own column of a shared-memory ring
// of 8 cells, and reads cells (including cell k-2 for the update) back from
// there.  Each thread touches only its own column, so no barrier is needed.
struct RowRing {
    double (*t)[8][kSweepThreads];  // [variable slot][ring position][thread]
    int tid;
    __device__ __forceinline__ double& at(int v, int k) { return t[v][k & 7][tid]; }
    __device__ __forceinline__ Cons cell(int k) {
        return Cons{at(0, k), at(Slots<1>::mn, k), at(Slots<1>::mt, k), at(3, k)};
    }
    // Cells [k, k+4) that are interior and <= kmax.
    __device__ __forceinline__ void fill(const SweepArgs& a, const LineGeom<1>& g, int k,
                                         int kmax, bool vec_ok) {
        const int lo = k > 2 ? k : 2;
        const int hi = min(min(k + 3, kmax), a.n - 3);
        if (vec_ok && lo == k && hi == k + 3) {
            const double* p = a.in + g.at(k);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const double2 x = __ldg(reinterpret_cast<const double2*>(p + v * a.vs));
                const double2 y = __ldg(reinterpret_cast<const double2*>(p + v * a.vs) + 1);
                at(v, k) = x.x;
                at(v, k + 1) = x.y;
                at(v, k + 2) = y.x;
                at(v, k + 3) = y.y;
            }
        } else {
            for (int kk = lo; kk <= hi; kk++) {
                const double* p = a.in + g.at(kk);
#pragma unroll
                for (int v = 0; v < 4; v++) at(v, kk) = __ldg(p + v * a.vs);
            }
        }
    }
};

// Column staging of the y sweep for stage sets with S::async_ring.  Each
// thread copies the interior cell AHEAD rows ahead of its column into its own
// column of a shared-memory ring with cp.async, so the load's latency hides
// behind AHEAD iterations of arithmetic without holding registers; cell k-2
// of the update is read back from the ring.  Slots hold cells k-2 .. k+AHEAD:
// 4 slots for AHEAD = 1, 8 up to AHEAD = 5; the copy of k+AHEAD reuses the
// slot of a cell no longer needed.  Each thread touches only its own column,
// so no barrier is needed.
template <int RW, int AHEAD>
struct ColumnRing {
    static_assert(AHEAD >= 1 && AHEAD <= 5, "ring depth");
    static constexpr int kSlots = AHEAD + 3 <= 4 ? 4 : 8;
    double (*t)[kSlots][RW];  // [variable][ring position][thread]
    int tid;
    __device__ __forceinline__ void issue(const SweepArgs& a, const LineGeom<2>& g, int k) {
        const double* p = a.in + g.at(k);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const unsigned dst =
                (unsigned)__cvta_generic_to_shared(&t[v][k & (kSlots - 1)][tid]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst),
                         "l"(p + v * a.vs)
                         : "memory");
        }
    }
    __device__ __forceinline__ void commit() {
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // Every group but the AHEAD most recent ones has landed.
    __device__ __forceinline__ void wait_ahead() {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(AHEAD) : "memory");
    }
    __device__ __forceinline__ Cons cell(int k) const {
        constexpr int mn = Slots<2>::mn, mt = Slots<2>::mt;
        const int q = k & (kSlots - 1);
        return Cons{t[0][q][tid], t[mn][q][tid], t[mt][q][tid], t[3][q][tid]};
    }
};

// The march of one thread over [k0, k1); S::Prim / S::Flux are the stage set's
// primitive and flux records, S::Sound what its primitives step hands to its
// trace step (the sound speed, with reciprocals in the mixed set).
// RW: threads of the CTA (the width of the y sweep's column ring).
template <int DIR, class S, int RW = kSweepThreads>
__device__ __forceinline__ void march(const SweepArgs& a, const typename S::Consts& C,
                                      const LineGeom<DIR>& g, int k0, int k1, double dtdx,
                                      double& cx, double& cy) {
    using Prim = typename S::Prim;
    using Flux = typename S::Flux;
    using Sound = typename S::Sound;
    const typename S::TraceK K = S::trace_constants(C, dtdx);

    __shared__ double ring_mem[DIR == 1 ? 4 : 1][8][kSweepThreads];
    RowRing ring{ring_mem, (int)threadIdx.x};
    // 16-byte loads need every address in + base + k + v*vs (in doubles) of a
    // chunk to be even from a 16-byte aligned pointer: aligned `in`, even
    // variable stride, even row start and an even first cell (chunks advance
    // by 4 cells).
    const bool vec_ok = DIR == 1 && ((reinterpret_cast<uintptr_t>(a.in) & 15) == 0) &&
                        ((a.vs & 1) == 0) && ((g.base & 1) == 0) && (((k0 - 2) & 1) == 0);

    Prim q1 = S::zero_prim(), q2 = S::zero_prim();  // primitives of k-1, k-2
    Sound c1 = S::zero_sound();                     // sound speed of k-1
    Prim xm2 = S::zero_prim();                      // qxm of k-2
    Flux fprev = S::zero_flux();                    // flux at (k-3 | k-2)

    // y sweep of a stage set with S::async_ring: the next cell is copied one
    // iteration ahead into the shared-memory column ring, so its latency hides
    // behind this iteration's arithmetic without holding registers.
    constexpr bool aring = DIR == 2 && S::async_ring;
    constexpr int ahead = aring ? S::ring_ahead : 1;
    using Ring = ColumnRing<aring ? RW : 1, ahead>;
    __shared__ double col_mem[aring ? 4 : 1][Ring::kSlots][aring ? RW : 1];
    Ring col{col_mem, (int)threadIdx.x};
    if (aring) {
        // Interior cells only (ghosts take the fused fill); one group per row,
        // empty for the rows not copied, so that the group count stays in step.
        for (int d = 0; d < ahead; d++) {
            const int kk = k0 - 2 + d;
            if (kk >= 2 && kk < a.n - 2 && kk <= k1 + 1)
                col.issue(a, reinterpret_cast<const LineGeom<2>&>(g), kk);
            col.commit();
        }
    }
    for (int k = k0 - 2; k <= k1 + 1; k++) {
        Cons uk;
        Cons u2{0.0, 0.0, 0.0, 0.0};
        if (aring) {
            const int kn = k + ahead;
            if (kn <= k1 + 1 && kn >= 2 && kn < a.n - 2)
                col.issue(a, reinterpret_cast<const LineGeom<2>&>(g), kn);
            col.commit();
            col.wait_ahead();
            uk = (k >= 2 && k < a.n - 2) ? col.cell(k) : load_cell<DIR>(a, g, k);
        } else if (DIR == 1) {
            if (((k - (k0 - 2)) & 3) == 0) ring.fill(a, reinterpret_cast<const LineGeom<1>&>(g), k,
                                                     k1 + 1, vec_ok);
            uk = (k >= 2 && k < a.n - 2) ? ring.cell(k) : load_cell<DIR>(a, g, k);
        } else {
            uk = load_cell<DIR>(a, g, k);
        }
        Prim qk;
        Sound ck;
        S::prim(C, uk, qk, ck);
        Prim xm1 = xm2;
        Flux f = fprev;
        if (k >= k0) {
            Prim dq = S::zero_prim();
            if (S::second_order(C)) S::slope4(C, q2, q1, qk, dq);
            Prim xp1;
            S::trace(K, q1, dq, c1, xm1, xp1);
            if (k >= k0 + 1) {
                f = S::riemann(C, xm2, xp1);
                if (k >= k0 + 2) {
                    if (DIR == 1) u2 = ring.cell(k - 2);
                    else if (aring) u2 = col.cell(k - 2);
                    // Otherwise cell k-2 is read again (a cache hit) instead of
                    // being carried in registers.
                    else u2 = load_interior<DIR>(a, g, k - 2);
                    const Cons o = S::update(u2, fprev, f, dtdx);
                    store_cell<DIR>(a, g, k - 2, o);
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
        }
        q2 = q1;
        q1 = qk;
        c1 = ck;
        xm2 = xm1;
        fprev = f;
    }
}

// The sweep kernel body: line and segment from the launch grid, dt from the
// device clock or the argument, fused Courant reduction.
template <int DIR, class S>
__device__ __forceinline__ void sweep_body(const SweepArgs& a, const Phys& P) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int segi = a.w_lo + (int)blockIdx.y;
    bool active = l < a.nlines && segi < a.w_hi;
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;
    if (active) {
        const typename S::Consts C = S::consts(P);
        const LineGeom<DIR> g(a, l);
        const double dtdx = dt / P.dx;
        const int k0 = 2 + segi * a.seg;
        const int k1 = min(k0 + a.seg, a.n - 2);
        march<DIR, S>(a, C, g, k0, k1, dtdx, cx, cy);
    }
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}


// ---------------------------------------------------------------------------
// The x sweep with one cell per lane.  A warp takes 32 consecutive cells
// [c - 2, c + 30) of one row, so every load and store instruction covers
// whole 128-byte lines of the row; neighbours are exchanged with warp
// shuffles instead of a marching window.  Lanes 2..29 produce the updates of
// cells [c, c + 28): the halo costs 4 of 32 lanes of arithmetic, against
// whole-line DRAM traffic (a row-marching thread consumes a line over many
// iterations and loses it from L2 in between).
template <class T>
__device__ __forceinline__ T shfl_up1(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <class T>
__device__ __forceinline__ T shfl_down1(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }

template <class P>
__device__ __forceinline__ P prim_up(const P& q) {
    return P{shfl_up1(q.r), shfl_up1(q.u), shfl_up1(q.v), shfl_up1(q.p)};
}
template <class P>
__device__ __forceinline__ P prim_down(const P& q) {
    return P{shfl_down1(q.r), shfl_down1(q.u), shfl_down1(q.v), shfl_down1(q.p)};
}
template <class F>
__device__ __forceinline__ F flux_up(const F& f) {
    return F{shfl_up1(f.d), shfl_up1(f.mn), shfl_up1(f.mt), shfl_up1(f.e)};
}


// One warp's window: line `row` (DIR 1: a row; DIR 2: a column, with lanes
// along y), output cells [c, c + 28) n [2, n - 2) with c = 28 * win, computed
// from cells [c - 2, c + 30) (one per lane).  Along x, windows start at
// multiples of 28 cells (7 sectors of 4 doubles), so when the row pitch is a
// multiple of 4 cells no 32-byte sector is written by two warps.  Accumulates
// the fused Courant maxima of its outputs into cx, cy.  The caller guarantees
// the warp is converged and `row` < a.nlines.
template <class S, int DIR>
__device__ __forceinline__ void line_window_1(const SweepArgs& a, const typename S::Consts& C,
                                              int row, int win, double dtdx, double& cx,
                                             double& cy) {
    using Prim = typename S::Prim;
    using Flux = typename S::Flux;
    using Sound = typename S::Sound;
    const int lane = threadIdx.x & 31;
    const int c = win * kCellWarpOut;                // first output cell of the warp
    if (c >= a.n - 2) return;                        // warp-uniform
    const int k = c - 2 + lane;                      // this lane's cell
    const LineGeom<DIR> g(a, row);
    const typename S::TraceK K = S::trace_constants(C, dtdx);
    const bool inside = k >= 0 && k < a.n;           // lanes outside the row idle
    const Cons u = inside ? load_cell<DIR>(a, g, k) : Cons{1.0, 0.0, 0.0, 1.0};
    Prim q;
    Sound cs;
    S::prim(C, u, q, cs);
    const Prim qm = prim_up(q), qp = prim_down(q);
    Prim dq = S::zero_prim();
    if (S::second_order(C)) S::slope4(C, qm, q, qp, dq);
    Prim xm, xp;
    S::trace(K, q, dq, cs, xm, xp);
    const Prim xp_next = prim_down(xp);              // qxp of cell k + 1
    const Flux f = S::riemann(C, xm, xp_next);       // interface (k | k + 1)
    const Flux f_prev = flux_up(f);                  // interface (k - 1 | k)
    if (lane >= 2 && lane < 2 + kCellWarpOut && k >= 2 && k < a.n - 2) {
        const Cons o = S::update(u, f_prev, f, dtdx);
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

template <class S>
__device__ __forceinline__ void xcell_window_1(const SweepArgs& a, const typename S::Consts& C,
                                             int row, int win, double dtdx, double& cx,
                                             double& cy) {
    line_window_1<S, 1>(a, C, row, win, dtdx, cx, cy);
}

// The same with two cells per lane: lane l holds cells ka = c - 2 + 2l and
// kb = ka + 1 of a 64-cell window, c = 60 * win, and lanes 1..30 produce the
// outputs [c, c + 60) (15 sectors).  The window's halo costs 4 of 64 cells
// instead of 4 of 32, and each shuffle of primitives, traces or fluxes serves
// two cells.  Every cell gets the same stage calls on the same inputs as in
// xcell_window_1.
// The window's arithmetic on this lane's two cells ka = c - 2 + 2 lane and
// kb = ka + 1 (ua, ub), already loaded.
template <class S>
__device__ __forceinline__ void xcell_window_2_cells(const SweepArgs& a,
                                                     const typename S::Consts& C,
                                                     const LineGeom<1>& g, int c, const Cons& ua,
                                                     const Cons& ub, double dtdx, double& cx,
                                                     double& cy) {
    using Prim = typename S::Prim;
    using Flux = typename S::Flux;
    using Sound = typename S::Sound;
    const int lane = threadIdx.x & 31;
    const int ka = c - 2 + 2 * lane, kb = ka + 1;
    const typename S::TraceK K = S::trace_constants(C, dtdx);
    Prim qa, qb;
    Sound ca, cb;
    S::prim(C, ua, qa, ca);
    S::prim(C, ub, qb, cb);
    const Prim qm = prim_up(qb), qp = prim_down(qa);  // cells ka - 1, kb + 1
    Prim dqa = S::zero_prim(), dqb = S::zero_prim();
    if (S::second_order(C)) {
        S::slope4(C, qm, qa, qb, dqa);
        S::slope4(C, qa, qb, qp, dqb);
    }
    Prim xma, xpa, xmb, xpb;
    S::trace(K, qa, dqa, ca, xma, xpa);
    S::trace(K, qb, dqb, cb, xmb, xpb);
    const Flux fab = S::riemann(C, xma, xpb);         // interface (ka | kb)
    const Prim xpn = prim_down(xpa);                  // qxp of kb + 1
    const Flux fbn = S::riemann(C, xmb, xpn);         // interface (kb | kb + 1)
    const Flux fpa = flux_up(fbn);                    // interface (ka - 1 | ka)
    if (lane >= 1 && lane <= 30) {
        if (ka >= 2 && ka < a.n - 2) {
            const Cons o = S::update(ua, fpa, fab, dtdx);
            store_cell<1>(a, g, ka, o);
            if (a.courant) {
                double cn, ct;
                S::courant(C, o, cn, ct);
                cx = cx > cn ? cx : cn;
                cy = cy > ct ? cy : ct;
            }
        }
        if (kb >= 2 && kb < a.n - 2) {
            const Cons o = S::update(ub, fab, fbn, dtdx);
            store_cell<1>(a, g, kb, o);
            if (a.courant) {
                double cn, ct;
                S::courant(C, o, cn, ct);
                cx = cx > cn ? cx : cn;
                cy = cy > ct ? cy : ct;
            }
        }
    }
}

// A cell of the two-cell window: loaded (with the fused boundary fill for
// ghosts), or a placeholder beyond the line that no output reads.
__device__ __forceinline__ Cons window_cell(const SweepArgs& a, const LineGeom<1>& g, int k) {
    return (k >= 0 && k < a.n) ? load_cell<1>(a, g, k) : Cons{1.0, 0.0, 0.0, 1.0};
}

template <class S>
__device__ __forceinline__ void xcell_window_2(const SweepArgs& a, const typename S::Consts& C,
                                               int row, int win, double dtdx, double& cx,
                                               double& cy) {
    const int lane = threadIdx.x & 31;
    const int c = win * kCellWarpOut2;               // first output cell of the warp
    if (c >= a.n - 2) return;                        // warp-uniform
    const int ka = c - 2 + 2 * lane;                 // this lane's two cells: ka, ka + 1
    const LineGeom<1> g(a, row);
    const Cons ua = window_cell(a, g, ka), ub = window_cell(a, g, ka + 1);
    xcell_window_2_cells<S>(a, C, g, c, ua, ub, dtdx, cx, cy);
}

// Software-pipelined runs of two-cell windows: while a window computes, the
// interior cells of the next one are copied into the other half of the warp's
// shared-memory stage.  Two ways to copy:
//  - WindowStage: each lane copies its own two cells with cp.async and reads
//    back only those, so no barrier is needed;
//  - BulkWindowStage: lane 0 copies each variable's interior span with one
//    bulk copy of the TMA engine (cp.async.bulk), completing on the buffer's
//    mbarrier, on which the warp waits.
// A stage row holds 66 cells: a bulk copy starts at the 16-byte boundary at or
// below the window's first interior cell, so the row may start one cell early.
constexpr int kStageRow = 66;
// Windows copied ahead of the one computing, and the stage's buffers (two
// windows ahead measured no faster: 4096^2 x sweep 0.250 ms either way).
constexpr int kStageAhead = 1;
constexpr int kStageBufs = kStageAhead + 1;
struct alignas(16) WindowStageMem {
    double t[kStageBufs][4][kStageRow];   // [buffer][variable][cell of the window (+ shift)]
    unsigned long long bar[kStageBufs];   // the bulk copies' mbarriers, one per buffer
};

struct WindowStage {
    WindowStageMem* m;
    __device__ __forceinline__ void begin() const {}
    __device__ __forceinline__ void end() const {}
    __device__ __forceinline__ void issue(const SweepArgs& a, const LineGeom<1>& g, int c,
                                          int b) const {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int k = c - 2 + 2 * lane + e;
            if (k >= 2 && k < a.n - 2) {
                const double* p = a.in + g.at(k);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const unsigned dst =
                        (unsigned)__cvta_generic_to_shared(&m->t[b][v][2 * lane + e]);
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst),
                                 "l"(p + v * a.vs)
                                 : "memory");
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    __device__ __forceinline__ void skip() const {
        asm volatile("cp.async.commit_group;\n" ::: "memory");  // an empty group
    }
    // Window t's copies have landed: every group but the kStageAhead most
    // recent ones.
    __device__ __forceinline__ void wait(int) const {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kStageAhead) : "memory");
    }
    __device__ __forceinline__ Cons cell(const SweepArgs& a, const LineGeom<1>& g, int c, int k,
                                         int b) const {
        if (k >= 2 && k < a.n - 2) {
            const int i = k - (c - 2);
            return Cons{m->t[b][0][i], m->t[b][Slots<1>::mn][i], m->t[b][Slots<1>::mt][i],
                        m->t[b][3][i]};
        }
        return window_cell(a, g, k);
    }
};

// Waits on a bulk copy's mbarrier that gave up (a copy that never completed);
// the host reads and clears the count (hydro_b200_domain_synchronize).
static __device__ unsigned int g_stage_wait_timeouts;
constexpr int kStageWaitSpins = 1 << 20;  // bounded: each try_wait suspends briefly

struct BulkWindowStage {
    WindowStageMem* m;
    __device__ __forceinline__ unsigned bar(int b) const {
        return (unsigned)__cvta_generic_to_shared(&m->bar[b]);
    }
    // Before the run's first copy / after its last wait: the warp's barriers
    // (4 arrivals a phase, one per variable's copy) are set up and torn down
    // by lane 0, with no copy in flight.
    __device__ __forceinline__ void begin() const {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {
            for (int b = 0; b < kStageBufs; b++)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;\n" ::"r"(bar(b)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncwarp();
    }
    __device__ __forceinline__ void end() const {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) {
            for (int b = 0; b < kStageBufs; b++)
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar(b)) : "memory");
        }
        __syncwarp();
    }
    // Cell shift of variable v's stage row: 1 when the variable's row starts
    // on an odd 8-byte slot (the copy then starts one cell early): the parity
    // of the state's base slot, plus the row offset's, plus v times the
    // variable stride's.
    __device__ __forceinline__ static int shift(const SweepArgs& a, const LineGeom<1>& g, int v) {
        return ((int)(reinterpret_cast<uintptr_t>(a.in) >> 3) + (int)g.base + v * (int)a.vs) & 1;
    }
    // The window at c: cells kA = max(c - 2, 2) .. kB = min(c + 61, n - 3) of
    // each variable, from the 16-byte boundary at or below cell kA (one cell
    // early when shift() is 1; kA is even), rounded up to whole 16 bytes (at
    // most cell kB + 1 <= n - 2, in the row).  Row position kA - (c - 2) is
    // even, so the destination is 16-byte aligned.  Lane v copies variable v.
    __device__ __forceinline__ void issue(const SweepArgs& a, const LineGeom<1>& g, int c,
                                          int b) const {
        __syncwarp();  // every lane has read the buffer's previous window
        const int v = threadIdx.x & 31;
        if (v < 4) {
            const int kA = c - 2 > 2 ? c - 2 : 2;
            const int kB = c + 61 < a.n - 3 ? c + 61 : a.n - 3;
            const int d = shift(a, g, v);
            const double* src = a.in + g.at(kA) + v * a.vs - d;
            const unsigned bytes = ((unsigned)(kB - kA + 1 + d) * 8u + 15u) & ~15u;
            const unsigned dst = (unsigned)__cvta_generic_to_shared(&m->t[b][v][kA - (c - 2)]);
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar(b)),
                         "r"(bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                "[%0], [%1], %2, [%3];\n" ::"r"(dst),
                "l"(src), "r"(bytes), "r"(bar(b))
                : "memory");
        }
    }
    __device__ __forceinline__ void skip() const {}
    // Window t's copies have landed: buffer t % kStageBufs completes its
    // (t / kStageBufs)-th phase.
    __device__ __forceinline__ void wait(int t) const {
        const unsigned addr = bar(t % kStageBufs), parity = (unsigned)(t / kStageBufs) & 1u;
        unsigned ok = 0;
        for (int i = 0; i < kStageWaitSpins && !ok; i++)
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                " selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(ok)
                : "r"(addr), "r"(parity)
                : "memory");
        if (!ok) atomicAdd(&g_stage_wait_timeouts, 1u);
    }
    __device__ __forceinline__ Cons cell(const SweepArgs& a, const LineGeom<1>& g, int c, int k,
                                         int b) const {
        if (k >= 2 && k < a.n - 2) {
            const int i = k - (c - 2);
            return Cons{m->t[b][0][i + shift(a, g, 0)],
                        m->t[b][Slots<1>::mn][i + shift(a, g, Slots<1>::mn)],
                        m->t[b][Slots<1>::mt][i + shift(a, g, Slots<1>::mt)],
                        m->t[b][3][i + shift(a, g, 3)]};
        }
        return window_cell(a, g, k);
    }
};

// One warp's windows win0 .. win0 + wins - 1 of rows row0 .. row0 + rows - 1
// (all valid), in row order, pipelined through the warp's stage.
template <class S, class Stage>
__device__ __forceinline__ void xpipe_run(const SweepArgs& a, const typename S::Consts& C,
                                          WindowStageMem* mem, int row0, int rows, int win0,
                                          int wins, double dtdx, double& cx, double& cy) {
    const Stage st{mem};
    const int lane = threadIdx.x & 31;
    const int n = rows * wins;
    st.begin();
    // Window t = r * wins + j; the copies run kStageAhead windows ahead.
    int ri = 0, ji = 0;  // the next window to copy
    for (int t = 0; t < kStageAhead; t++) {
        if (t < n) {
            st.issue(a, LineGeom<1>(a, row0 + ri), (win0 + ji) * kCellWarpOut2, t % kStageBufs);
            if (++ji == wins) ji = 0, ++ri;
        } else {
            st.skip();
        }
    }
    int r = 0, j = 0;  // the window to compute
    for (int t = 0; t < n; t++) {
        const int ti = t + kStageAhead;
        if (ti < n) {
            st.issue(a, LineGeom<1>(a, row0 + ri), (win0 + ji) * kCellWarpOut2, ti % kStageBufs);
            if (++ji == wins) ji = 0, ++ri;
        } else {
            st.skip();
        }
        st.wait(t);
        const int b = t % kStageBufs;
        const LineGeom<1> g(a, row0 + r);
        const int c = (win0 + j) * kCellWarpOut2;
        const int ka = c - 2 + 2 * lane;
        const Cons ua = st.cell(a, g, c, ka, b), ub = st.cell(a, g, c, ka + 1, b);
        xcell_window_2_cells<S>(a, C, g, c, ua, ub, dtdx, cx, cy);
        if (++j == wins) j = 0, ++r;
    }
    st.end();
}

// Grid: x = rows, y = ceil(runs of NW windows / warps per CTA).
template <class S, int NW, class Stage>
__device__ __forceinline__ void xpipe_body(const SweepArgs& a, const Phys& P) {
    __shared__ WindowStageMem stage_mem[kCellThreads / 32];
    const int warp = threadIdx.x >> 5;
    const int row = blockIdx.x;
    const int total = (a.n - 2 + kCellWarpOut2 - 1) / kCellWarpOut2;
    const int w0 = a.w_lo + (blockIdx.y * (blockDim.x >> 5) + warp) * NW;
    int w1 = w0 + NW;
    w1 = w1 < a.w_hi ? w1 : a.w_hi;
    w1 = w1 < total ? w1 : total;
    bool active = row < a.nlines && w0 < w1;
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;
    if (active) {
        const typename S::Consts C = S::consts(P);
        xpipe_run<S, Stage>(a, C, &stage_mem[warp], row, 1, w0, w1 - w0, dt / P.dx, cx, cy);
    }
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}

// The x-sweep window of a stage set (S::cells_per_lane); its outputs per
// warp are window_out<S>().
template <class S>
__device__ __forceinline__ void xcell_window(const SweepArgs& a, const typename S::Consts& C,
                                             int row, int win, double dtdx, double& cx,
                                             double& cy) {
    if constexpr (S::cells_per_lane == 2)
        xcell_window_2<S>(a, C, row, win, dtdx, cx, cy);
    else
        xcell_window_1<S>(a, C, row, win, dtdx, cx, cy);
}

// Grid: x = rows, y = ceil(windows / warps per CTA).
template <class S>
__device__ __forceinline__ void xcell_body(const SweepArgs& a, const Phys& P) {
    const int win = a.w_lo + blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int row = blockIdx.x;
    bool active = row < a.nlines && win < a.w_hi;
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;
    if (active) {
        const typename S::Consts C = S::consts(P);
        xcell_window<S>(a, C, row, win, dt / P.dx, cx, cy);
    }
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}

// The standalone Courant reduction (compute_deltat.c:54-73) over the interior
// of one state, with the stage set's per-cell formula so that it agrees with
// the reduction fused into the sweeps of the same precision.
template <class S>
__device__ __forceinline__ void courant_body(const double* __restrict__ u, int nx, int ny,
                                             int nxt, long long vs, const Phys& P,
                                             unsigned long long* cour_x,
                                             unsigned long long* cour_y) {
    const typename S::Consts C = S::consts(P);
    double cx = 0.0, cy = 0.0;
    const long long total = (long long)nx * ny;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / nx) + 2, i = (int)(c % nx) + 2;
        const long long o = i + (long long)nxt * j;
        const Cons w{__ldg(u + o), __ldg(u + o + vs), __ldg(u + o + 2 * vs), __ldg(u + o + 3 * vs)};
        double cn, ct;
        S::courant(C, w, cn, ct);
        cx = cx > cn ? cx : cn;
        cy = cy > ct ? cy : ct;
    }
    warp_max_atomic(cour_x, cx);
    warp_max_atomic(cour_y, cy);
}

}  // namespace hb
