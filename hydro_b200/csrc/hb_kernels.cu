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
#include "hb_march.cuh"
#include "hb_coop.cuh"
#include "hb_batch_body.cuh"

namespace hb {

template <int DIR, bool UNIT>
__global__ void __launch_bounds__(kSweepThreads, DIR == 2 ? kFp64MarchMinBlocks : 1)
sweep_kernel(const SweepArgs a, const Phys P) {
    sweep_body<DIR, ExactStages<UNIT>>(a, P);
}

template <bool UNIT>
__global__ void __launch_bounds__(kCellThreads, kFp64CellMinBlocks)
xcell_kernel(const SweepArgs a, const Phys P) {
    xcell_body<ExactStages<UNIT>>(a, P);
}

// The y sweep with one cell per lane (lanes along a column): for grids too
// small to fill the GPU with marching segments, every cell of a window is
// computed at once instead of one after another.  Same stage calls on the
// same inputs as the marcher, so the same bits.
template <bool UNIT>
__global__ void __launch_bounds__(kCellThreads, kFp64CellMinBlocks)
ycell_kernel(const SweepArgs a, const Phys P) {
    const int win = a.w_lo + blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int line = blockIdx.x;
    bool active = line < a.nlines && win < a.w_hi;
    double dt = a.dt;
    if (a.clk) {
        active = active && a.clk->active;
        dt = a.clk->dt;
    }
    double cx = 0.0, cy = 0.0;
    if (active) {
        const typename ExactStages<UNIT>::Consts C = ExactStages<UNIT>::consts(P);
        line_window_1<ExactStages<UNIT>, 2>(a, C, line, win, dt / P.dx, cx, cy);
    }
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}

cudaError_t launch_ycell(const SweepArgs& a, const Phys& P, cudaStream_t s) {
    const int nwin = window_span(a, (a.n - 2 + kCellWarpOut - 1) / kCellWarpOut);
    const int wpc = kCellThreads / 32;
    if (nwin == 0) return cudaSuccess;
    const dim3 grid(a.nlines, (nwin + wpc - 1) / wpc);
    if (P.unit_slope) ycell_kernel<true><<<grid, kCellThreads, 0, s>>>(a, P);
    else ycell_kernel<false><<<grid, kCellThreads, 0, s>>>(a, P);
    return cudaGetLastError();
}

// The cooperative window (hb_coop.cuh): a CTA of G warps per 32G cells of a
// line, register cap as the warp window's (kFp64CellMinBlocks CTAs of 64
// threads per SM).
template <bool UNIT, int DIR, int G>
__global__ void __launch_bounds__(32 * G, kFp64CellMinBlocks * 2 / G)
coop_kernel(const SweepArgs a, const Phys P) {
    coop_body<ExactStages<UNIT>, DIR, G>(a, P);
}

// The cooperative window over runs of NW windows per CTA, software-pipelined
// (coop_pipe_body).
template <bool UNIT, int DIR, int G, int NW>
__global__ void __launch_bounds__(32 * G, kFp64CoopPipeMinBlocks)
coop_pipe_kernel(const SweepArgs a, const Phys P) {
    coop_pipe_body<ExactStages<UNIT>, DIR, G, NW>(a, P);
}

template <int G>
static cudaError_t launch_coop_g(int dir, const SweepArgs& a, const Phys& P, cudaStream_t s) {
    const int nwin = window_span(a, coop_windows<G>(a.n));
    if (nwin == 0) return cudaSuccess;
    if constexpr (G == 4) {
        constexpr int NW = kFp64CoopPipeWindows;
        if (dir == 1 && coop_pipe_pays(a.nlines, nwin, device_sm_count())) {
            const dim3 pgrid(a.nlines, (nwin + NW - 1) / NW);
            if (P.unit_slope) coop_pipe_kernel<true, 1, G, NW><<<pgrid, 32 * G, 0, s>>>(a, P);
            else coop_pipe_kernel<false, 1, G, NW><<<pgrid, 32 * G, 0, s>>>(a, P);
            return cudaGetLastError();
        }
    }
    const dim3 grid(a.nlines, nwin);
    if (dir == 1) {
        if (P.unit_slope) coop_kernel<true, 1, G><<<grid, 32 * G, 0, s>>>(a, P);
        else coop_kernel<false, 1, G><<<grid, 32 * G, 0, s>>>(a, P);
    } else {
        if (P.unit_slope) coop_kernel<true, 2, G><<<grid, 32 * G, 0, s>>>(a, P);
        else coop_kernel<false, 2, G><<<grid, 32 * G, 0, s>>>(a, P);
    }
    return cudaGetLastError();
}

cudaError_t launch_coop(int dir, int warps, const SweepArgs& a, const Phys& P, cudaStream_t s) {
    if (warps == 8) return launch_coop_g<8>(dir, a, P, s);
    return launch_coop_g<4>(dir, a, P, s);
}

static dim3 xcell_grid(const SweepArgs& a) {
    // Windows [28w, 28w + 28) cover the outputs [2, n - 2).
    const int nwin = window_span(a, (a.n - 2 + kCellWarpOut - 1) / kCellWarpOut);
    const int wpc = kCellThreads / 32;
    return dim3(a.nlines, (nwin + wpc - 1) / wpc);
}

cudaError_t launch_xcell(const SweepArgs& a, const Phys& P, cudaStream_t s) {
    if (xcell_grid(a).y == 0) return cudaSuccess;
    if (P.unit_slope) xcell_kernel<true><<<xcell_grid(a), kCellThreads, 0, s>>>(a, P);
    else xcell_kernel<false><<<xcell_grid(a), kCellThreads, 0, s>>>(a, P);
    return cudaGetLastError();
}

cudaError_t launch_sweep(int dir, const SweepArgs& a, const Phys& P, cudaStream_t s) {
    const int nl = a.n - 4;
    const int nseg = window_span(a, (nl + a.seg - 1) / a.seg);
    if (nseg == 0) return cudaSuccess;
    dim3 grid((a.nlines + kSweepThreads - 1) / kSweepThreads, nseg);
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
    const int slot = cour_slot();
    courant_body<ExactStages<true>>(u, nx, ny, nxt, vs, P, &cour[slot], &cour[kCourSlots + slot]);
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

int device_sm_count() {
    // Cached per device: the attribute does not change while the process runs.
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
            return 1;
        cache[dev] = n;
    }
    return cache[dev];
}

cudaError_t launch_courant(const double* u, int nx, int ny, int nxt, long long vs, const Phys& P,
                           unsigned long long* cour, cudaStream_t s) {
    const long long total = (long long)nx * ny;
    long long blocks = (total + 255) / 256;
    const long long cap = 8ll * device_sm_count();  // 8 resident CTAs of 256 threads per SM
    if (blocks > cap) blocks = cap;
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

// Halo strips of a domain split (make_boundary.c:48-52, mpibounds.c:165-310):
// the two interior lines next to one side, for the interior lines of the other
// direction, packed as [var][line][2] (idim 1: columns, per interior row) or
// [var][2][line] (idim 2: rows, per interior column).  Pack reads interior
// cells of `u`; unpack writes the ghost cells of the same side.  One thread per
// value; the index map is the same both ways, so unpacking a neighbour's pack
// of the opposite side puts its cells where a single grid would have them.
__global__ void halo_kernel(double* u, double* buf, int pack, int idim, int side, int nx, int ny,
                            int nxt, long long vs) {
    const int nlines = (idim == 1) ? ny : nx;
    const int total = 8 * nlines;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int v, l, c;
    if (idim == 1) {
        c = t & 1;
        l = (t >> 1) % nlines;
        v = (t >> 1) / nlines;
    } else {
        l = t % nlines;
        c = (t / nlines) & 1;
        v = (t / nlines) >> 1;
    }
    const int nl = (idim == 1) ? nx : ny;
    // interior source line and ghost destination line along the sweep axis
    const int k_in = side == 0 ? 2 + c : nl + c;
    const int k_gh = side == 0 ? c : nl + 2 + c;
    const int k = pack ? k_in : k_gh;
    const long long at = (idim == 1) ? (long long)nxt * (l + 2) + k : (long long)nxt * k + (l + 2);
    if (pack)
        buf[t] = u[at + v * vs];
    else
        u[at + v * vs] = buf[t];
}

cudaError_t launch_halo(double* u, double* buf, int pack, int idim, int side, int nx, int ny,
                        int nxt, long long vs, cudaStream_t s) {
    const int nlines = (idim == 1) ? ny : nx;
    const int threads = 8 * nlines;
    halo_kernel<<<(threads + 255) / 256, 256, 0, s>>>(u, buf, pack, idim, side, nx, ny, nxt, vs);
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
        unsigned long long mx = 0ull, my = 0ull;
        for (int s = 0; s < kCourSlots; s++) {
            mx = cour[s] > mx ? cour[s] : mx;
            my = cour[kCourSlots + s] > my ? cour[kCourSlots + s] : my;
            cour[s] = 0ull;
            cour[kCourSlots + s] = 0ull;
        }
        const double cx = __longlong_as_double((long long)mx);
        const double cy = __longlong_as_double((long long)my);
        double dt = courant_factor * dx / omax(cx, omax(cy, smallc));
        if (c->nstep == 0) dt = dt / 2.0;
        c->dt = dt;
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

// ---------------------------------------------------------------- batches
template <bool UNIT, int DIR, int T>
__global__ void __launch_bounds__(T, (DIR == 1 ? kBatchXThreadsPerSm : kBatchYThreadsPerSm) / T)
batch_sweep_kernel(const BatchLaunch L, const Phys P) {
    batch_sweep_body<ExactStages<UNIT>, DIR, T>(L, P);
}

template <bool UNIT, int T>
static void launch_batch_t(const BatchLaunch& L, const Phys& P, int dir, int grid,
                           cudaStream_t s) {
    if (dir == 1) batch_sweep_kernel<UNIT, 1, T><<<grid, T, 0, s>>>(L, P);
    else batch_sweep_kernel<UNIT, 2, T><<<grid, T, 0, s>>>(L, P);
}

cudaError_t launch_batch_sweep(const BatchLaunch& L, const Phys& P, int dir, int grid,
                               cudaStream_t s) {
    if (L.threads == 128) {
        if (P.unit_slope) launch_batch_t<true, 128>(L, P, dir, grid, s);
        else launch_batch_t<false, 128>(L, P, dir, grid, s);
    } else {
        if (P.unit_slope) launch_batch_t<true, 64>(L, P, dir, grid, s);
        else launch_batch_t<false, 64>(L, P, dir, grid, s);
    }
    return cudaGetLastError();
}

template <class K>
static int occupancy(K kernel, int threads) {
    int n = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

template <bool UNIT, int T>
static int batch_occ(int dir) {
    return dir == 1 ? occupancy(batch_sweep_kernel<UNIT, 1, T>, T)
                    : occupancy(batch_sweep_kernel<UNIT, 2, T>, T);
}

int batch_sweep_blocks_per_sm_exact(bool unit_slope, int dir, int threads) {
    if (threads == 128) return unit_slope ? batch_occ<true, 128>(dir) : batch_occ<false, 128>(dir);
    return unit_slope ? batch_occ<true, 64>(dir) : batch_occ<false, 64>(dir);
}

// main.c:349-392 per instance (see clock_begin_kernel).
__global__ void batch_clock_begin_kernel(BatchInst* inst, int nslots, double courant_factor,
                                         double smallc, long long* gstep) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    BatchInst& I = inst[s];
    if (!I.active) return;
    if (!((I.t < I.tend) && (I.nstep < I.nstepmax))) {
        I.active = 0;
        I.stop_step = *gstep;
        return;
    }
    if ((I.nstep % 2) == 0) {
        unsigned long long mx = 0ull, my = 0ull;
        for (int k = 0; k < kBatchCourSlots; k++) {
            mx = I.cour[k] > mx ? I.cour[k] : mx;
            my = I.cour[kBatchCourSlots + k] > my ? I.cour[kBatchCourSlots + k] : my;
            I.cour[k] = 0ull;
            I.cour[kBatchCourSlots + k] = 0ull;
        }
        const double cx = __longlong_as_double((long long)mx);
        const double cy = __longlong_as_double((long long)my);
        double dt = courant_factor * I.dx / omax(cx, omax(cy, smallc));
        if (I.nstep == 0) dt = dt / 2.0;
        I.dt = dt;
    }
}

__global__ void batch_clock_end_kernel(BatchInst* inst, int nslots, long long* gstep) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) *gstep += 1;
    if (s >= nslots) return;
    BatchInst& I = inst[s];
    if (!I.active) return;
    I.nstep++;
    I.t += I.dt;
}

cudaError_t launch_batch_clock_begin(BatchInst* inst, int nslots, double courant_factor,
                                     double smallc, long long* gstep, cudaStream_t s) {
    batch_clock_begin_kernel<<<(nslots + 127) / 128, 128, 0, s>>>(inst, nslots, courant_factor,
                                                                  smallc, gstep);
    return cudaGetLastError();
}

cudaError_t launch_batch_clock_end(BatchInst* inst, int nslots, long long* gstep,
                                   cudaStream_t s) {
    batch_clock_end_kernel<<<(nslots + 127) / 128, 128, 0, s>>>(inst, nslots, gstep);
    return cudaGetLastError();
}

// Courant maxima of the listed instances (grid y: one instance per entry).
__global__ void __launch_bounds__(256)
batch_courant_kernel(BatchInst* inst, const int* slots, int nslots, Phys P) {
    batch_courant_body<ExactStages<true>>(inst, slots, nslots, P);
}

// A single-blast initial state written on the device: density rho, zero
// momenta and energy e_bg in the interior, ghost cells 0, and energy e_blast
// in the padded cell (bi, bj) -- the layout of hydro_funcs.c:15-112.
__global__ void blast_init_kernel(double* u, int nx, int ny, double rho, double ebg, int bi,
                                  int bj, double eblast) {
    const int nxt = nx + 4, nyt = ny + 4;
    const long long vs = (long long)nxt * nyt;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < vs;
         c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c / nxt), i = (int)(c % nxt);
        const bool in = i >= 2 && i < nx + 2 && j >= 2 && j < ny + 2;
        u[c] = in ? rho : 0.0;
        u[c + vs] = 0.0;
        u[c + 2 * vs] = 0.0;
        u[c + 3 * vs] = in ? ((i == bi && j == bj) ? eblast : ebg) : 0.0;
    }
}

cudaError_t launch_blast_init(double* u, int nx, int ny, double rho, double ebg, int bi, int bj,
                              double eblast, cudaStream_t s) {
    const long long vs = (long long)(nx + 4) * (ny + 4);
    long long blocks = (vs + 255) / 256;
    const long long cap = 16ll * device_sm_count();
    if (blocks > cap) blocks = cap;
    blast_init_kernel<<<(unsigned)blocks, 256, 0, s>>>(u, nx, ny, rho, ebg, bi, bj, eblast);
    return cudaGetLastError();
}

cudaError_t launch_batch_courant(BatchInst* inst, const int* slots, int nslots, const Phys& P,
                                 bool mixed, cudaStream_t s) {
    if (nslots <= 0) return cudaSuccess;
    if (mixed) return launch_batch_courant_mixed(inst, slots, nslots, P, s);
    batch_courant_kernel<<<dim3(16, nslots), 256, 0, s>>>(inst, slots, nslots, P);
    return cudaGetLastError();
}

}  // namespace hb
