// hb_fast.cu -- the sweep kernels of the FMA FP64 stage set
// (hb_stages_fast.cuh): the same skeletons as the bit-exact FP64 kernels
// (hb_march.cuh, hb_coop.cuh), built with FMA contraction.
#include "../../include/hydro_b200.h"
#include "hb_kernels.cuh"
#include "hb_march.cuh"
#include "hb_coop.cuh"
#include "hb_stages_fast.cuh"

namespace hb {

template <int DIR>
__global__ void __launch_bounds__(kSweepThreads, kFp64MarchMinBlocks)
sweep_fast_kernel(const SweepArgs a, const Phys P) {
    sweep_body<DIR, FastStages>(a, P);
}

// The warp window along rows (DIR 1) or columns (DIR 2).
template <int DIR>
__global__ void __launch_bounds__(kCellThreads, kFp64CellMinBlocks)
warp_fast_kernel(const SweepArgs a, const Phys P) {
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
        const FastStages::Consts C = FastStages::consts(P);
        line_window_1<FastStages, DIR>(a, C, line, win, dt / P.dx, cx, cy);
    }
    if (a.courant) {
        const int slot = cour_slot();
        warp_max_atomic(&a.courant[slot], cx);
        warp_max_atomic(&a.courant[kCourSlots + slot], cy);
    }
}

template <int DIR, int G>
__global__ void __launch_bounds__(32 * G, kFp64CellMinBlocks * 2 / G)
coop_fast_kernel(const SweepArgs a, const Phys P) {
    coop_body<FastStages, DIR, G>(a, P);
}

// The x window over software-pipelined runs (as the bit-exact set's).
__global__ void __launch_bounds__(128, kFp64CoopPipeMinBlocks)
coop_pipe_fast_kernel(const SweepArgs a, const Phys P) {
    coop_pipe_body<FastStages, 1, 4, kFp64CoopPipeWindows>(a, P);
}

cudaError_t launch_sweep_fast(int dir, int kernel, const SweepArgs& a, const Phys& P,
                              cudaStream_t s) {
    if (kernel == HB_KERNEL_WARP) {
        const int nwin = window_span(a, (a.n - 2 + kCellWarpOut - 1) / kCellWarpOut);
        const int wpc = kCellThreads / 32;
        if (nwin == 0) return cudaSuccess;
        const dim3 grid(a.nlines, (nwin + wpc - 1) / wpc);
        if (dir == 1) warp_fast_kernel<1><<<grid, kCellThreads, 0, s>>>(a, P);
        else warp_fast_kernel<2><<<grid, kCellThreads, 0, s>>>(a, P);
    } else if (kernel == HB_KERNEL_COOP) {
        const int nwin = window_span(a, coop_windows<4>(a.n));
        if (nwin == 0) return cudaSuccess;
        if (dir == 1 && coop_pipe_pays(a.nlines, nwin, device_sm_count())) {
            const dim3 pgrid(a.nlines, (nwin + kFp64CoopPipeWindows - 1) / kFp64CoopPipeWindows);
            coop_pipe_fast_kernel<<<pgrid, 128, 0, s>>>(a, P);
            return cudaGetLastError();
        }
        const dim3 grid(a.nlines, nwin);
        if (dir == 1) coop_fast_kernel<1, 4><<<grid, 128, 0, s>>>(a, P);
        else coop_fast_kernel<2, 4><<<grid, 128, 0, s>>>(a, P);
    } else if (kernel == HB_KERNEL_COOP8) {
        const int nwin = window_span(a, coop_windows<8>(a.n));
        if (nwin == 0) return cudaSuccess;
        const dim3 grid(a.nlines, nwin);
        if (dir == 1) coop_fast_kernel<1, 8><<<grid, 256, 0, s>>>(a, P);
        else coop_fast_kernel<2, 8><<<grid, 256, 0, s>>>(a, P);
    } else {
        const int nl = a.n - 4;
        const int nseg = window_span(a, (nl + a.seg - 1) / a.seg);
        if (nseg == 0) return cudaSuccess;
        const dim3 grid((a.nlines + kSweepThreads - 1) / kSweepThreads, nseg);
        if (dir == 1) sweep_fast_kernel<1><<<grid, kSweepThreads, 0, s>>>(a, P);
        else sweep_fast_kernel<2><<<grid, kSweepThreads, 0, s>>>(a, P);
    }
    return cudaGetLastError();
}

int sweep_fast_blocks_per_sm(int dir) {
    int n = 0;
    cudaError_t e = dir == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                   &n, sweep_fast_kernel<1>, kSweepThreads, 0)
                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                   &n, sweep_fast_kernel<2>, kSweepThreads, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

__global__ void __launch_bounds__(256)
courant_fast_kernel(const double* __restrict__ u, int nx, int ny, int nxt, long long vs, Phys P,
                    unsigned long long* cour) {
    const int slot = cour_slot();
    courant_body<FastStages>(u, nx, ny, nxt, vs, P, &cour[slot], &cour[kCourSlots + slot]);
}

cudaError_t launch_courant_fast(const double* u, int nx, int ny, int nxt, long long vs,
                                const Phys& P, unsigned long long* cour, cudaStream_t s) {
    const long long total = (long long)nx * ny;
    long long blocks = (total + 255) / 256;
    const long long cap = 8ll * device_sm_count();  // 8 resident CTAs of 256 threads per SM
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    courant_fast_kernel<<<(unsigned)blocks, 256, 0, s>>>(u, nx, ny, nxt, vs, P, cour);
    return cudaGetLastError();
}

}  // namespace hb
