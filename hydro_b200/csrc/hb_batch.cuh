// hb_batch.cuh -- many independent HydroC runs advanced together.
//
// A batch holds up to `capacity` instances ("slots"), each a grid of its own
// size with its own state, scratch buffer, clock (t, dt, nstep) and Courant
// accumulators, all resident in one device arena.  One global step advances
// every active instance by one time step of its own (main.c:344-408 per
// instance): a clock kernel (dt on even steps, stop test), two persistent
// sweep launches that pull work items of all instances from a queue, and a
// clock kernel (t += dt, nstep++).  Warps claim work items from a queue: an x
// item is a run of cell windows of one row, or of several rows of a narrow
// grid (cell-per-lane x sweep); a y item is a group of 32 columns (one per
// lane) over one row segment (marching y sweep).  Instances need not share the
// sweep order: each instance's first sweep is x on its even steps
// and y on its odd ones, so the host builds two item lists from the
// instances' step parities and the launches alternate them.  A list holds no
// record per item: it is a run per instance (its first item's index and its
// item counts), and a warp decodes the item it claims from its index, so the
// host's cost of building a list grows with the instances, not with the cells.
#pragma once

#include "hb_kernels.cuh"

namespace hb {

struct BatchInst {
    double* A;          // state, reference layout
    double* B;          // scratch of the same size (first sweep's output)
    int nx, ny, nxt, nyt;
    long long vs;
    int bnd_left, bnd_right, bnd_down, bnd_up;
    double dx;
    double t, dt, tend;
    int nstep, nstepmax;
    int active;         // 1 while t < tend and nstep < nstepmax (0 for free slots)
    int pad0;
    // Courant maxima of the current state (bit patterns): kBatchCourSlots slots
    // of max(c+|u|) then kBatchCourSlots of max(c+|v|), the slot chosen by the
    // CTA, so that large instances do not funnel every warp's atomic into one
    // address; readers take the max over the slots.
    unsigned long long cour[2 * 16];
    long long stop_step;         // global step at which the instance stopped (-1: running)
};

// One warp's work: an x item is `wins` consecutive cell windows from window
// k0 of each of `rows` consecutive rows (narrow grids pack several rows into
// one item); a y item is 32 columns from `line` marching the row segment that
// starts at output row k0.
struct WorkItem {
    int slot;
    int line;  // x: first interior row; y: first interior column of the group
    int k0;    // x: first cell window; y: first output cell (row) of the segment
    int rows;  // x: rows of the item (1 for y)
    int wins;  // x: windows per row (0 for y)
};

// The items of one instance in one list, numbered from `first` in the list:
//  - x, a grid of at least XW = x_item_windows() windows per row: `per` items
//    per row, item j covers row j / per, windows from (j % per) * XW;
//  - x, a narrower grid: per = -(rows per item), item j covers rows from
//    j * rows, all `nwin` windows of each;
//  - y: `per` row segments per column group, item j is group j / per
//    (kBatchYItemColumns columns), segment j % per.
struct ItemRun {
    int slot;
    int per;
    int nwin;   // x: cell windows per row
    int pad;
};

// Threads per CTA of the batched sweep (the autotuner's "threads per tile"):
// 64 or 128.  Each warp of a CTA claims its own items, so no CTA barrier sits
// between items; a y item is a group of kBatchYItemColumns columns over one
// row segment, one per lane.  Narrow grids waste fewer lanes with 32-column
// groups: on the seeded 256-instance mix (sides 64..1024) 3.1% of y lanes
// idle, against 8.0% with 64.
constexpr int kBatchThreadChoices[2] = {64, 128};
constexpr int kBatchYItemColumns = 32;
constexpr int kBatchCourSlots = 16; // Courant accumulator slots per instance
// Resident threads per SM the item kernels are compiled for (register caps,
// as minimum CTAs per SM = threads / CTA size), measured on the 256-instance
// batch:
//  - FP64 x items: 896 (72 registers); uncapped (96 registers) they are
//    latency-bound, and 14 CTAs of 64 are 5% faster per step than 10.
//  - FP64 y items: 1024, the plain FP64 march's cap (64 registers): 134
//    registers uncapped, 15% slower per batched step.
//  - mixed x items: 512 (121 registers), pipelined (below).
//  - mixed y items (marching, cp.async column ring): 448; uncapped they take 147
//    registers (6 CTAs of 64), 7 CTAs of 64 are 3% faster, 8 less so.
// The caps need not match the single-grid kernels': no stage set rounds
// differently in another kernel (the FP64 set rounds every operation once,
// the mixed set writes its fused multiply-adds out), so batched instances
// equal their single-grid runs bit for bit under any cap or CTA size.
constexpr int kBatchXThreadsPerSm = 896;
constexpr int kBatchYThreadsPerSm = 1024;
constexpr int kBatchXMixedThreadsPerSm = 512;
// Mixed x items run their windows software-pipelined (xpipe_run, at 512
// threads per SM: 121 registers), in items of up to 12 two-cell windows.  On
// the 256-instance batch (G cell-steps/s): 28.52 so, 28.33 with items of 8,
// 27.40 with items of 4; with plain loads at 768 threads per SM, 27.82 (items
// of 4) and 28.29 (items of 8).
constexpr bool kBatchXPipe = true;
constexpr int kBatchYMixedThreadsPerSm = 448;
// Cell windows per x item (one warp's): FP64 (one cell per lane) 4, mixed
// (two cells per lane, pipelined) 12.
__host__ __device__ constexpr int x_item_windows(bool two_cell) { return two_cell ? 12 : 4; }

struct BatchLaunch {
    BatchInst* inst;
    const ItemRun* runs;       // one per instance with items in this list
    const int* run_first;      // list index of each run's first item (ascending, from 0)
    int nruns;
    int nitems;                // items in the list (all runs)
    int phase;                 // 1: A -> B (first sweep of the step), 2: B -> A
    unsigned int* counter;     // claim counter, zero before the launch
    int seg;                   // y-segment length used to build the items
    int claim;                 // items a warp claims per atomic
    int threads;               // threads per CTA (one of kBatchThreadChoices)
};

// Launchers (hb_kernels.cu for FP64, hb_mixed.cu for the mixed form).
// One launch sweeps the items of one direction (dir 1: x, 2: y) with
// L.threads threads per CTA.
cudaError_t launch_batch_sweep(const BatchLaunch& L, const Phys& P, int dir, int grid,
                               cudaStream_t s);
cudaError_t launch_batch_sweep_mixed(const BatchLaunch& L, const Phys& P, int dir, int grid,
                                     cudaStream_t s);
int batch_sweep_blocks_per_sm(bool mixed, bool unit_slope, int dir, int threads);
cudaError_t launch_batch_clock_begin(BatchInst* inst, int nslots, double courant_factor,
                                     double smallc, long long* gstep, cudaStream_t s);
cudaError_t launch_batch_clock_end(BatchInst* inst, int nslots, long long* gstep,
                                   cudaStream_t s);
cudaError_t launch_blast_init(double* u, int nx, int ny, double rho, double ebg, int bi, int bj,
                              double eblast, cudaStream_t s);
// Courant maxima of the listed instances' current states (slot per entry),
// with the per-cell formula of the batch's precision.
cudaError_t launch_batch_courant(BatchInst* inst, const int* slots, int nslots, const Phys& P,
                                 bool mixed, cudaStream_t s);
cudaError_t launch_batch_courant_mixed(BatchInst* inst, const int* slots, int nslots,
                                       const Phys& P, cudaStream_t s);

}  // namespace hb
