// hb_kernels.cu -- the fused FP64 sweep kernel and its companions.
//
// One launch performs one dimension-split sweep (hydro_godunov.c:70-139 for
// one idim) over every interior line.  Each thread owns one line segment and
// marches along it, carrying a five-cell window in registers:
//
//   load cell k (fused make_boundary for ghost cells)  -> constoprim + EOS
//   slope + trace of cell k-1                          -> qxm, qxp
//   riemann + cmpflx at the interface (k-2 | k-1)      -> flux
//   update of cell k-2 with the fluxes on its two faces -> store
//
// so every intermediate array of the reference (u, q, c, e, dq, qxm, qxp,
// qleft, qright, qgdnv, flux, and the riemann scratch) lives in registers and
// HBM sees only the state: 4 doubles read and 4 written per cell and sweep
// (plus a 4-cell halo per segment).  Threads of a warp own adjacent lines, so
// in the y sweep (lines = columns) every load and store instruction covers 32
// consecutive doubles of a row.  In the x sweep (lines = rows) each thread
// walks its own row; consecutive loads of a thread fall in the same 32-byte
// sector and are served from L1.
//
// The sweep reads `in` and writes `out` (two buffers), so segments of one
// line can run in parallel without the read-before-overwrite hazard of the
// reference's in-place update; the host alternates the buffers so the state
// ends in the resident array after both sweeps.
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

__device__ __forceinline__ void warp_max_atomic(unsigned long long* dst, double v) {
    for (int o = 16; o > 0; o >>= 1) v = omax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

template <int DIR, bool UNIT>
__global__ void __launch_bounds__(kSweepThreads)
sweep_kernel(const SweepArgs a, const Phys P) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = l < a.nlines;
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;  // fused Courant maxima of this thread
    if (active) {
        const LineGeom<DIR> g(a, l);
        const double dtdx = dt / P.dx;
        const TraceK K = trace_constants(P.scheme, dtdx);
        const int k0 = 2 + blockIdx.y * a.seg;
        const int k1 = min(k0 + a.seg, a.n - 2);

        Prim q1, q2;        // primitives of k-1, k-2
        double c1 = 0.0;    // sound speed of k-1
        Prim xm2;           // qxm of k-2
        Cons fprev;         // flux at (k-3 | k-2)
        q1 = q2 = xm2 = Prim{0.0, 0.0, 0.0, 0.0};
        fprev = Cons{0.0, 0.0, 0.0, 0.0};

        for (int k = k0 - 2; k <= k1 + 1; k++) {
            const Cons uk = load_cell<DIR>(a, g, k);
            Prim qk;
            double ck;
            cons_to_prim(P, uk, qk, ck);
            Prim xm1 = xm2;
            Cons f = fprev;
            if (k >= k0) {
                Prim dq{0.0, 0.0, 0.0, 0.0};
                if (P.iorder != 1) slope4<UNIT>(P.slope_type, q2, q1, qk, dq);
                Prim xp1;
                trace1(K, q1, dq, c1, xm1, xp1);
                if (k >= k0 + 1) {
                    f = riemann_flux(P, xm2, xp1);
                    if (k >= k0 + 2) {
                        // Cell k-2 is interior: its conservative values are read
                        // again (an L1/L2 hit) instead of being carried.
                        const Cons u2 = load_interior<DIR>(a, g, k - 2);
                        const Cons o = update(u2, fprev, f, dtdx);
                        store_cell<DIR>(a, g, k - 2, o);
                        if (a.courant) {
                            double cn, ct;
                            courant_speeds(P, o, cn, ct);
                            if (DIR == 1) {
                                cx = omax(cx, cn);
                                cy = omax(cy, ct);
                            } else {
                                cx = omax(cx, ct);
                                cy = omax(cy, cn);
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
    if (a.courant) {
        warp_max_atomic(&a.courant[0], cx);
        warp_max_atomic(&a.courant[1], cy);
    }
}

cudaError_t launch_sweep(int dir, const SweepArgs& a, const Phys& P, cudaStream_t s) {
    const int nl = a.n - 4;
    dim3 grid((a.nlines + kSweepThreads - 1) / kSweepThreads, (nl + a.seg - 1) / a.seg);
    if (dir == 1) {
        if (P.unit_slope) sweep_kernel<1, true><<<grid, kSweepThreads, 0, s>>>(a, P);
        else sweep_kernel<1, false><<<grid, kSweepThreads, 0, s>>>(a, P);
    } else {
        if (P.unit_slope) sweep_kernel<2, true><<<grid, kSweepThreads, 0, s>>>(a, P);
        else sweep_kernel<2, false><<<grid, kSweepThreads, 0, s>>>(a, P);
    }
    return cudaGetLastError();
}

// compute_deltat.c:54-73 as one pass over the interior: Courant speeds of
// every cell (ComputeQEforRow + equation_of_state + courantOnXY), max-reduced
// per warp and merged with atomicMax on the bit patterns (c + |u| >= 0, so
// the unsigned order of the patterns is the numeric order and max is exact).
__global__ void __launch_bounds__(256)
courant_kernel(const double* __restrict__ u, int nx, int ny, int nxt, long long vs, Phys P,
               unsigned long long* cour) {
    double cx = 0.0, cy = 0.0;
    const long long total = (long long)nx * ny;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / nx) + 2, i = (int)(c % nx) + 2;
        const long long o = i + (long long)nxt * j;
        Cons w{__ldg(u + o), __ldg(u + o + vs), __ldg(u + o + 2 * vs), __ldg(u + o + 3 * vs)};
        double cn, ct;
        courant_speeds(P, w, cn, ct);
        cx = omax(cx, cn);
        cy = omax(cy, ct);
    }
    warp_max_atomic(&cour[0], cx);
    warp_max_atomic(&cour[1], cy);
}

int sweep_blocks_per_sm(int dir, bool unit_slope) {
    int n = 0;
    cudaError_t e;
    if (dir == 1)
        e = unit_slope ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_kernel<1, true>,
                                                                       kSweepThreads, 0)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_kernel<1, false>,
                                                                       kSweepThreads, 0);
    else
        e = unit_slope ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_kernel<2, true>,
                                                                       kSweepThreads, 0)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_kernel<2, false>,
                                                                       kSweepThreads, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

cudaError_t launch_courant(const double* u, int nx, int ny, int nxt, long long vs, const Phys& P,
                           unsigned long long* cour, cudaStream_t s) {
    const long long total = (long long)nx * ny;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    courant_kernel<<<(unsigned)blocks, 256, 0, s>>>(u, nx, ny, nxt, vs, P, cour);
    return cudaGetLastError();
}

// make_boundary.c:53-198 on its own (the sweeps fuse it): one thread per
// (interior line, ghost layer) of direction idim, all four variables.
__global__ void boundary_kernel(double* u, int idim, int nx, int ny, int nxt, int nyt,
                                long long vs, int bnd_lo, int bnd_hi) {
    const int nlines = (idim == 1) ? ny : nx;
    const int n = (idim == 1) ? nxt : nyt;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nlines * 4) return;
    const int l = t >> 2, gidx = t & 3;
    const int k = gidx < 2 ? gidx : n - 4 + gidx;
    const int bt = gidx < 2 ? bnd_lo : bnd_hi;
    int src;
    long long base, step;
    int mn;
    if (idim == 1) {
        src = ghost_source<1>(bt, k, n);
        base = (long long)nxt * (l + 2);
        step = 1;
        mn = 1;
    } else {
        src = ghost_source<2>(bt, k, n);
        base = l + 2;
        step = nxt;
        mn = 2;
    }
    if (src < 0) return;
    const double sn = (bt == 1) ? -1.0 : 1.0;
    for (int s = 0; s < 4; s++)
        u[base + step * k + s * vs] = u[base + step * src + s * vs] * (s == mn ? sn : 1.0);
}

cudaError_t launch_boundary(double* u, int idim, int nx, int ny, int nxt, int nyt, long long vs,
                            int bnd_lo, int bnd_hi, cudaStream_t s) {
    const int nlines = (idim == 1) ? ny : nx;
    const int threads = nlines * 4;
    boundary_kernel<<<(threads + 127) / 128, 128, 0, s>>>(u, idim, nx, ny, nxt, nyt, vs, bnd_lo,
                                                          bnd_hi);
    return cudaGetLastError();
}

// main.c:349-392 on the device: on even steps dt = courant_factor*dx /
// MAX(cournox, MAX(cournoy, smallc)), halved at step 0; stops the clock once
// t >= tend or nstep >= nstepmax.  Resets the Courant accumulators for the
// reduction fused into the next odd step.
__global__ void clock_begin_kernel(DevClock* c, unsigned long long* cour, double courant_factor,
                                   double dx, double smallc) {
    if (!c->active) return;
    if (!((c->t < c->tend) && (c->nstep < c->nstepmax))) {
        c->active = 0;
        return;
    }
    if ((c->nstep % 2) == 0) {
        const double cx = __longlong_as_double((long long)cour[0]);
        const double cy = __longlong_as_double((long long)cour[1]);
        double dt = courant_factor * dx / omax(cx, omax(cy, smallc));
        if (c->nstep == 0) dt = dt / 2.0;
        c->dt = dt;
        cour[0] = 0ull;
        cour[1] = 0ull;
    }
}

// main.c:407-408: nstep++, t += dt (and the dt record).
__global__ void clock_end_kernel(DevClock* c) {
    if (!c->active) return;
    const int idx = c->nstep - c->nstep0;
    if (c->dts && idx >= 0 && idx < c->ndts) c->dts[idx] = c->dt;
    c->nstep++;
    c->t += c->dt;
}

cudaError_t launch_clock_begin(DevClock* c, unsigned long long* cour, double courant_factor,
                               double dx, double smallc, cudaStream_t s) {
    clock_begin_kernel<<<1, 1, 0, s>>>(c, cour, courant_factor, dx, smallc);
    return cudaGetLastError();
}

cudaError_t launch_clock_end(DevClock* c, cudaStream_t s) {
    clock_end_kernel<<<1, 1, 0, s>>>(c);
    return cudaGetLastError();
}

}  // namespace hb
