// hb_batch_body.cuh -- the persistent batched sweep (device side), templated
// on the stage set.  Included by hb_kernels.cu (FP64) and hb_mixed.cu (mixed).
#pragma once

#include "hb_batch.cuh"
#include "hb_march.cuh"

namespace hb {

__device__ __forceinline__ SweepArgs batch_args(const BatchInst& I, int dir, int phase,
                                                bool fuse, BatchInst* Ip) {
    SweepArgs a;
    a.in = phase == 1 ? I.A : I.B;
    a.out = phase == 1 ? I.B : I.A;
    a.resid = I.A;
    a.gout = I.A;
    a.clk = nullptr;
    a.dt = I.dt;
    a.courant = fuse ? Ip->cour : nullptr;
    a.nx = I.nx;
    a.ny = I.ny;
    a.nxt = I.nxt;
    a.nyt = I.nyt;
    a.vs = I.vs;
    if (dir == 1) {
        a.bnd_lo = I.bnd_left;
        a.bnd_hi = I.bnd_right;
        a.nlines = I.ny;
        a.n = I.nxt;
    } else {
        a.bnd_lo = I.bnd_down;
        a.bnd_hi = I.bnd_up;
        a.nlines = I.nx;
        a.n = I.nyt;
    }
    a.seg = 0;
    a.w_lo = 0;
    a.w_hi = kWholeLine;
    return a;
}

// The run holding list item `it`: the last run whose first item is <= it.
// The warp searches together, 32 candidates a round (two rounds cover 1024
// runs); run 0 starts at item 0, so lane 0's candidate always qualifies.
__device__ __forceinline__ int find_run(const int* first, int nruns, int it, int lane) {
    int lo = 0, n = nruns;
    while (n > 1) {
        const int step = (n + 31) >> 5;
        const bool ok = lane * step < n && __ldg(first + lo + lane * step) <= it;
        const int k = 31 - __clz(__ballot_sync(0xffffffffu, ok));
        lo += k * step;
        n = min(step, n - k * step);
    }
    return lo;
}

// Item `it` of the list, from its run (ItemRun); XW windows per x item.
// `run` carries the warp's last run from claim to claim: consecutive claims
// mostly fall in it.
template <int DIR, int XW>
__device__ __forceinline__ WorkItem decode_item(const BatchLaunch& L, int it, int lane, int& run) {
    const bool hit = run >= 0 && __ldg(L.run_first + run) <= it &&
                     (run + 1 == L.nruns || it < __ldg(L.run_first + run + 1));
    if (!hit) run = find_run(L.run_first, L.nruns, it, lane);
    const ItemRun R = L.runs[run];
    const int j = it - __ldg(L.run_first + run);
    WorkItem w;
    w.slot = R.slot;
    if (DIR == 2) {
        w.line = (j / R.per) * kBatchYItemColumns;
        w.k0 = 2 + (j % R.per) * L.seg;
        w.rows = 1;
        w.wins = 0;
    } else if (R.per > 0) {
        w.line = j / R.per;
        w.k0 = (j % R.per) * XW;
        w.rows = 1;
        w.wins = min(XW, R.nwin - w.k0);
    } else {
        w.line = j * -R.per;
        w.k0 = 0;
        w.rows = -R.per;   // clipped to the grid's rows by the caller
        w.wins = R.nwin;
    }
    return w;
}

// Persistent warps claim `claim` items at a time (lane 0 takes them with one
// atomic and broadcasts the base) until the list is exhausted, so warps never
// wait for each other.  Every item of the list sweeps direction DIR, so each
// direction has its own kernel with its own register budget.  An item's
// instance is skipped once its clock has stopped.  The second sweep of an
// instance's odd step also reduces its Courant maxima.
template <class S, int DIR, int T>
__device__ __forceinline__ void batch_sweep_body(const BatchLaunch& L, const Phys& P) {
    const typename S::Consts C = S::consts(P);
    const int lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * (T / 32) + (threadIdx.x >> 5);
    // The pipelined x items' stage (WindowStageMem: kStageBufs windows of two
    // cells per lane, per warp).
    constexpr bool xpipe = DIR == 1 && S::cells_per_lane == 2 && kBatchXPipe;
    __shared__ WindowStageMem stage_mem[xpipe ? T / 32 : 1];
    int run = -1;
    for (;;) {
        int base = 0;
        if (lane == 0) base = (int)atomicAdd(L.counter, (unsigned)L.claim);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= L.nitems) break;
        const int end = min(base + L.claim, L.nitems);
        for (int it = base; it < end; it++) {
            constexpr int XW = x_item_windows(S::cells_per_lane == 2);
            const WorkItem w = decode_item<DIR, XW>(L, it, lane, run);
            BatchInst* Ip = L.inst + w.slot;
            const BatchInst I = *Ip;
            if (!I.active) continue;  // warp-uniform
            const bool fuse = (L.phase == 2) && (I.nstep & 1);
            const SweepArgs a = batch_args(I, DIR, L.phase, fuse, Ip);
            const double dtdx = I.dt / I.dx;
            double cx = 0.0, cy = 0.0;
            if (DIR == 1) {
                const int rows = min(w.rows, I.ny - w.line);
                if constexpr (xpipe) {
                    xpipe_run<S, WindowStage>(a, C, &stage_mem[threadIdx.x >> 5], w.line, rows,
                                              w.k0, w.wins, dtdx, cx, cy);
                } else {
                    for (int r = 0; r < rows; r++)
                        for (int j = 0; j < w.wins; j++)
                            xcell_window<S>(a, C, w.line + r, w.k0 + j, dtdx, cx, cy);
                }
            } else {
                const int l = w.line + lane;
                if (l < a.nlines) {
                    const LineGeom<2> g(a, l);
                    const int k1 = min(w.k0 + L.seg, a.n - 2);
                    march<2, S, T>(a, C, g, w.k0, k1, dtdx, cx, cy);
                }
            }
            if (fuse) {
                const int slot = gwarp % kBatchCourSlots;
                warp_max_atomic(&Ip->cour[slot], cx);
                warp_max_atomic(&Ip->cour[kBatchCourSlots + slot], cy);
            }
        }
    }
}

// The standalone Courant maxima of listed batch instances (grid y = entry).
template <class S>
__device__ __forceinline__ void batch_courant_body(BatchInst* inst, const int* slots, int nslots,
                                                   const Phys& P) {
    const int e = blockIdx.y;
    if (e >= nslots) return;
    BatchInst* Ip = inst + slots[e];
    const int slot = blockIdx.x % kBatchCourSlots;
    courant_body<S>(Ip->A, Ip->nx, Ip->ny, Ip->nxt, Ip->vs, P, &Ip->cour[slot],
                    &Ip->cour[kBatchCourSlots + slot]);
}

}  // namespace hb
