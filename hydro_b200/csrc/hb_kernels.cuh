// hb_kernels.cuh -- kernel argument records and launchers shared by the
// host runtime (hb_runtime.cu) and the kernels (hb_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hb_stages.cuh"

namespace hb {

// Device-resident clock of the multi-step driver (main.c:344-408 state).
struct DevClock {
    double t, dt, tend;
    int nstep, nstepmax;
    int nstep0;   // nstep when the clock was last set (index base of dts)
    int active;   // 0 once t >= tend or nstep >= nstepmax
    double* dts;  // optional per-step dt record
    int ndts;
};

// One fused sweep over every interior line of a direction.
struct SweepArgs {
    const double* in;        // interior cells are read here
    const double* resid;     // the resident state: ghost cells are read (and sourced) here
                             // when they are not interior cells
    double* out;             // updated interior cells are written here
    double* gout;            // ghost cells of the swept direction are written here (or null)
    const DevClock* clk;     // null: use dt below; else dt and the active flag come from here
    double dt;
    unsigned long long* courant;  // null or [2 * kCourSlots] fused maxima (bit patterns)
    int nx, ny, nxt, nyt;
    long long vs;            // nxt * nyt (stride between variables)
    int bnd_lo, bnd_hi;      // boundary types of the swept direction (left/right or down/up)
    int seg;                 // output cells per thread segment
    int nlines;              // interior lines (ny for the x sweep, nx for the y sweep)
    int n;                   // cells along a line including ghosts (nxt or nyt)
    // Windows (segments for the marching kernels) [w_lo, w_hi) of every line
    // are swept: the launch grid starts at window w_lo.  0 and a large w_hi
    // sweep the whole line; a domain split sweeps the windows that read no
    // ghost cell while the halos travel, and the others after.
    int w_lo, w_hi;
};

// Windows of [w_lo, w_hi) n [0, total) a launch covers (its grid's y extent
// in windows; 0: nothing to launch).
inline int window_span(const SweepArgs& a, int total) {
    const int hi = a.w_hi < total ? a.w_hi : total;
    return hi > a.w_lo ? hi - a.w_lo : 0;
}
constexpr int kWholeLine = 1 << 30;  // w_hi of a launch over whole lines

constexpr int kSweepThreads = 64;

// The fused Courant maxima are accumulated with atomicMax into kCourSlots
// slots per direction ([0, kCourSlots): max(c+|u|), [kCourSlots, 2*kCourSlots):
// max(c+|v|)), the slot chosen by the CTA index, so that no single address
// takes one atomic per warp of the whole grid; readers take the max over the
// slots (max is exact, so the result does not depend on the split).
constexpr int kCourSlots = 128;

// Multiprocessor count of the current device (cudaDevAttrMultiProcessorCount,
// cached per device; 1 if it cannot be read).
int device_sm_count();

// Launchers (hb_kernels.cu).  Each returns the cudaError_t of the launch.
cudaError_t launch_sweep(int dir, const SweepArgs& a, const Phys& P, cudaStream_t s);
// Resident sweep CTAs per SM (cudaOccupancyMaxActiveBlocksPerMultiprocessor).
int sweep_blocks_per_sm(int dir, bool unit_slope);
// The x sweep with one cell per lane (hb_march.cuh xcell_body): FP64 and mixed.
constexpr int kCellThreads = 64;

// Minimum resident CTAs per SM the sweep kernels are compiled for (register
// caps).  The FP64 kernels are latency-bound: more resident warps beat the
// few register spills the caps cause (measured at 4096^2: marching y sweep
// 1.66 -> 1.49 ms, cell-per-lane x sweep 1.63 -> 1.56 ms).  The mixed marching
// sweep is not capped; the mixed x sweep (two cells per lane) runs best at 12
// CTAs per SM (80 registers): 0.419 ms at 4096^2, against 0.477 ms one cell
// per lane.
constexpr int kFp64MarchMinBlocks = 16;
constexpr int kFp64CellMinBlocks = 18;
constexpr int kMixedCellMinBlocks = 12;
// The software-pipelined mixed x sweep (xpipe_body): two-cell windows per warp
// and its register cap (8 CTAs of 64 per SM: 119 registers, no spills).  At
// 4096^2: 0.258 ms with runs of 6 windows, 0.267 with 8, 0.268 with 4, 0.304
// with 2 (at 12 CTAs per SM and 80 registers, runs of 4: 0.291 ms), against
// 0.309 ms for one window per warp.
constexpr int kMixedXPipeWindows = 6;
constexpr int kMixedXPipeMinBlocks = 8;
// The FP64 cooperative x window (4 warps) over software-pipelined runs of
// windows per CTA (coop_pipe_body), used when the runs make at least four
// waves of resident CTAs, and its minimum CTAs of 128 threads per SM.  At
// 4096^2 (34 windows a row): 0.744 ms with runs of 8, 0.752 of 4, 0.759 of 12,
// 0.778 of 2, 0.780 of 17, 0.813 of 34, against 0.782 ms one window per CTA.
constexpr int kFp64CoopPipeWindows = 8;
constexpr int kFp64CoopPipeMinBlocks = 9;
// Whether a cooperative x launch over `nwin` windows of `nlines` lines takes
// pipelined runs (host side; sm_count from device_sm_count()).
inline bool coop_pipe_pays(long long nlines, int nwin, int sm_count) {
    return nlines * ((nwin + kFp64CoopPipeWindows - 1) / kFp64CoopPipeWindows) >=
           4LL * sm_count * kFp64CoopPipeMinBlocks;
}
constexpr int kCellWarpOut = 28;   // outputs per warp of the cell-per-lane x sweep
constexpr int kCellWarpOut2 = 60;  // the same with two cells per lane
// Outputs per warp of the x sweep window of a stage set.
template <class S>
constexpr int window_out() { return S::cells_per_lane == 2 ? kCellWarpOut2 : kCellWarpOut; }
cudaError_t launch_xcell(const SweepArgs& a, const Phys& P, cudaStream_t s);
// The cooperative window (hb_coop.cuh), `warps` = 4 or 8 warps per CTA.
cudaError_t launch_coop(int dir, int warps, const SweepArgs& a, const Phys& P, cudaStream_t s);
cudaError_t launch_coop_mixed(int dir, int warps, const SweepArgs& a, const Phys& P,
                              cudaStream_t s);
cudaError_t launch_ycell(const SweepArgs& a, const Phys& P, cudaStream_t s);
// The mixed x sweep (two-cell windows); `bulk`: staged by TMA-engine bulk
// copies (HB_KERNEL_BULK) instead of per-lane cp.async.
cudaError_t launch_xcell_mixed(const SweepArgs& a, const Phys& P, cudaStream_t s,
                               bool bulk = false);
// Waits of the mixed x sweep's bulk-copy stage that gave up (hb_mixed.cu).
int mixed_stage_wait_timeouts(bool reset);
// The FMA FP64 stage set (hb_fast.cu): kernel = HB_KERNEL_* (include/hydro_b200.h).
cudaError_t launch_sweep_fast(int dir, int kernel, const SweepArgs& a, const Phys& P,
                              cudaStream_t s);
int sweep_fast_blocks_per_sm(int dir);
cudaError_t launch_courant_fast(const double* u, int nx, int ny, int nxt, long long vs,
                                const Phys& P, unsigned long long* cour, cudaStream_t s);
// The mixed-precision sweep (hb_mixed.cu).
cudaError_t launch_sweep_mixed(int dir, const SweepArgs& a, const Phys& P, cudaStream_t s);
int sweep_mixed_blocks_per_sm(int dir);
cudaError_t launch_courant(const double* u, int nx, int ny, int nxt, long long vs, const Phys& P,
                           unsigned long long* cour, cudaStream_t s);
cudaError_t launch_courant_mixed(const double* u, int nx, int ny, int nxt, long long vs,
                                 const Phys& P, unsigned long long* cour, cudaStream_t s);
cudaError_t launch_boundary(double* u, int idim, int nx, int ny, int nxt, int nyt, long long vs,
                            int bnd_lo, int bnd_hi, cudaStream_t s);
cudaError_t launch_vtk_base64(const double* var_plane, int nx, int ny, int nxt,
                              unsigned char* out, cudaStream_t s);
cudaError_t launch_halo(double* u, double* buf, int pack, int idim, int side, int nx, int ny,
                        int nxt, long long vs, cudaStream_t s);
cudaError_t launch_clock_begin(DevClock* c, unsigned long long* cour, double courant_factor,
                               double dx, double smallc, cudaStream_t s);
cudaError_t launch_clock_end(DevClock* c, cudaStream_t s);

}  // namespace hb
