// hb_mixed.cu -- the mixed-precision sweep kernel (stage set in
// hb_stages_mixed.cuh, march skeleton in hb_march.cuh).  Built with fast FP32
// division / square root and no FMA contraction: the stage code writes its
// fused multiply-adds out (see the Makefile).
#include "hb_kernels.cuh"
#include "hb_march.cuh"
#include "hb_coop.cuh"
#include "hb_stages_mixed.cuh"
#include "hb_batch_body.cuh"

namespace hb {

template <int DIR>
__global__ void __launch_bounds__(kSweepThreads)
sweep_mixed_kernel(const SweepArgs a, const Phys P) {
    sweep_body<DIR, MixedStages>(a, P);
}

__global__ void __launch_bounds__(kCellThreads, kMixedCellMinBlocks)
xcell_mixed_kernel(const SweepArgs a, const Phys P) {
    xcell_body<MixedStages>(a, P);
}

template <int NW, class Stage>
__global__ void __launch_bounds__(kCellThreads, kMixedXPipeMinBlocks)
xpipe_mixed_kernel(const SweepArgs a, const Phys P) {
    xpipe_body<MixedStages, NW, Stage>(a, P);
}

// Waits on the bulk-copy stage's mbarriers that gave up since the last call
// (g_stage_wait_timeouts of this translation unit), cleared when `reset`;
// -1 if the count cannot be read.
int mixed_stage_wait_timeouts(bool reset) {
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, g_stage_wait_timeouts, sizeof v) != cudaSuccess) return -1;
    if (v && reset) {
        const unsigned z = 0;
        if (cudaMemcpyToSymbol(g_stage_wait_timeouts, &z, sizeof z) != cudaSuccess) return -1;
    }
    return (int)v;
}

// The x sweep: runs of kMixedXPipeWindows pipelined windows per warp when
// they make at least four waves of the pipelined kernel's resident warps,
// else one window per warp (small grids need the parallelism more).  `bulk`
// always takes the pipelined runs, staged by bulk copies.
cudaError_t launch_xcell_mixed(const SweepArgs& a, const Phys& P, cudaStream_t s, bool bulk) {
    const int nwin =
        window_span(a, (a.n - 2 + window_out<MixedStages>() - 1) / window_out<MixedStages>());
    const int wpc = kCellThreads / 32;
    if (nwin == 0) return cudaSuccess;
    constexpr int NW = kMixedXPipeWindows;
    const long long runs = (long long)a.nlines * ((nwin + NW - 1) / NW);
    const dim3 pgrid(a.nlines, ((nwin + NW - 1) / NW + wpc - 1) / wpc);
    if (bulk) {
        xpipe_mixed_kernel<NW, BulkWindowStage><<<pgrid, kCellThreads, 0, s>>>(a, P);
        return cudaGetLastError();
    }
    if (runs >= 4LL * device_sm_count() * kMixedXPipeMinBlocks * wpc) {
        xpipe_mixed_kernel<NW, WindowStage><<<pgrid, kCellThreads, 0, s>>>(a, P);
        return cudaGetLastError();
    }
    dim3 grid(a.nlines, (nwin + wpc - 1) / wpc);
    xcell_mixed_kernel<<<grid, kCellThreads, 0, s>>>(a, P);
    return cudaGetLastError();
}

// The cooperative window (hb_coop.cuh) with the mixed stage set, at the warp
// window's thread count per SM (kMixedCellMinBlocks CTAs of 64 threads).
template <int DIR, int G>
__global__ void __launch_bounds__(32 * G, kMixedCellMinBlocks * 2 / G)
coop_mixed_kernel(const SweepArgs a, const Phys P) {
    coop_body<MixedStages, DIR, G>(a, P);
}

template <int G>
static cudaError_t launch_coop_mixed_g(int dir, const SweepArgs& a, const Phys& P,
                                       cudaStream_t s) {
    const int nwin = window_span(a, coop_windows<G>(a.n));
    if (nwin == 0) return cudaSuccess;
    const dim3 grid(a.nlines, nwin);
    if (dir == 1) coop_mixed_kernel<1, G><<<grid, 32 * G, 0, s>>>(a, P);
    else coop_mixed_kernel<2, G><<<grid, 32 * G, 0, s>>>(a, P);
    return cudaGetLastError();
}

cudaError_t launch_coop_mixed(int dir, int warps, const SweepArgs& a, const Phys& P,
                              cudaStream_t s) {
    if (warps == 8) return launch_coop_mixed_g<8>(dir, a, P, s);
    return launch_coop_mixed_g<4>(dir, a, P, s);
}

cudaError_t launch_sweep_mixed(int dir, const SweepArgs& a, const Phys& P, cudaStream_t s) {
    const int nl = a.n - 4;
    const int nseg = window_span(a, (nl + a.seg - 1) / a.seg);
    if (nseg == 0) return cudaSuccess;
    dim3 grid((a.nlines + kSweepThreads - 1) / kSweepThreads, nseg);
    if (dir == 1)
        sweep_mixed_kernel<1><<<grid, kSweepThreads, 0, s>>>(a, P);
    else
        sweep_mixed_kernel<2><<<grid, kSweepThreads, 0, s>>>(a, P);
    return cudaGetLastError();
}

int sweep_mixed_blocks_per_sm(int dir) {
    int n = 0;
    cudaError_t e = dir == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                   &n, sweep_mixed_kernel<1>, kSweepThreads, 0)
                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                   &n, sweep_mixed_kernel<2>, kSweepThreads, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

template <int DIR, int T>
__global__ void __launch_bounds__(T, (DIR == 1 ? kBatchXMixedThreadsPerSm
                                               : kBatchYMixedThreadsPerSm) / T)
batch_sweep_mixed_kernel(const BatchLaunch L, const Phys P) {
    batch_sweep_body<MixedStages, DIR, T>(L, P);
}

cudaError_t launch_batch_sweep_mixed(const BatchLaunch& L, const Phys& P, int dir, int grid,
                                     cudaStream_t s) {
    if (L.threads == 128) {
        if (dir == 1) batch_sweep_mixed_kernel<1, 128><<<grid, 128, 0, s>>>(L, P);
        else batch_sweep_mixed_kernel<2, 128><<<grid, 128, 0, s>>>(L, P);
    } else {
        if (dir == 1) batch_sweep_mixed_kernel<1, 64><<<grid, 64, 0, s>>>(L, P);
        else batch_sweep_mixed_kernel<2, 64><<<grid, 64, 0, s>>>(L, P);
    }
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256)
courant_mixed_kernel(const double* __restrict__ u, int nx, int ny, int nxt, long long vs, Phys P,
                     unsigned long long* cour) {
    const int slot = cour_slot();
    courant_body<MixedStages>(u, nx, ny, nxt, vs, P, &cour[slot], &cour[kCourSlots + slot]);
}

cudaError_t launch_courant_mixed(const double* u, int nx, int ny, int nxt, long long vs,
                                 const Phys& P, unsigned long long* cour, cudaStream_t s) {
    const long long total = (long long)nx * ny;
    long long blocks = (total + 255) / 256;
    const long long cap = 8ll * device_sm_count();  // 8 resident CTAs of 256 threads per SM
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    courant_mixed_kernel<<<(unsigned)blocks, 256, 0, s>>>(u, nx, ny, nxt, vs, P, cour);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256)
batch_courant_mixed_kernel(BatchInst* inst, const int* slots, int nslots, Phys P) {
    batch_courant_body<MixedStages>(inst, slots, nslots, P);
}

cudaError_t launch_batch_courant_mixed(BatchInst* inst, const int* slots, int nslots,
                                       const Phys& P, cudaStream_t s) {
    batch_courant_mixed_kernel<<<dim3(16, nslots), 256, 0, s>>>(inst, slots, nslots, P);
    return cudaGetLastError();
}

int batch_sweep_blocks_per_sm_exact(bool unit_slope, int dir, int threads);  // hb_kernels.cu

template <int T>
static int batch_mixed_occ(int dir) {
    int n = 0;
    cudaError_t e = dir == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                   &n, batch_sweep_mixed_kernel<1, T>, T, 0)
                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                   &n, batch_sweep_mixed_kernel<2, T>, T, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

int batch_sweep_blocks_per_sm(bool mixed, bool unit_slope, int dir, int threads) {
    if (!mixed) return batch_sweep_blocks_per_sm_exact(unit_slope, dir, threads);
    return threads == 128 ? batch_mixed_occ<128>(dir) : batch_mixed_occ<64>(dir);
}

}  // namespace hb
