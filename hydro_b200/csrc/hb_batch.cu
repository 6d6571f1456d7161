// hb_batch.cu -- host side of batches (hb_batch.cuh): the device arena that
// holds every instance's state and scratch, the slot table, the work-item
// lists, the CUDA graphs of one global step, and the tile autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hydro_b200.h"
#include "hb_batch.cuh"

int hb_record_error(int code, const char* msg);  // hb_runtime.cu

using hb::BatchInst;
using hb::BatchLaunch;
using hb::ItemRun;

namespace {

int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
    char buf[384];
    if (e != cudaSuccess)
        snprintf(buf, sizeof(buf), "batch: %s: %s", what, cudaGetErrorString(e));
    else
        snprintf(buf, sizeof(buf), "batch: %s", what);
    return hb_record_error(code, buf);
}

#define HB_BCU(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? HB_ERR_NOMEM : HB_ERR_CUDA, #call, \
                        e_);                                                              \
    } while (0)

struct Tuning {
    int seg = 64;          // y-segment length of y items
    int claim = 1;         // items a warp claims at a time
    int blocks_per_sm = 0; // persistent CTAs per SM (0: occupancy limit)
    int threads = 64;      // threads per CTA (columns per y item)
};

std::mutex g_tune_mu;
std::map<std::string, Tuning> g_tune_cache;  // shape signature -> best tiling

// First-fit allocator over the arena, in units of 32 doubles (256 bytes).
struct Arena {
    double* base = nullptr;
    long long units = 0;
    std::map<long long, long long> free_;  // offset -> length (units)
    void init(double* b, long long u) {
        base = b;
        units = u;
        free_.clear();
        if (u > 0) free_[0] = u;
    }
    long long alloc(long long n) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                const long long off = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[off + n] = len - n;
                return off;
            }
        }
        return -1;
    }
    void release(long long off, long long n) {
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    long long free_units() const {
        long long s = 0;
        for (auto& kv : free_) s += kv.second;
        return s;
    }
};

}  // namespace

struct hb_batch {
    int capacity = 0;
    int precision = HB_PREC_MIXED;
    hb::Phys P{};
    double courant_factor = 0.8;
    cudaStream_t stream = nullptr;
    int device = 0, sm_count = 0;  // cudaDevAttrMultiProcessorCount, read at creation
    // slots
    std::vector<BatchInst> h;        // host copy of the table
    std::vector<long long> off;      // arena offset (units) of each slot, -1 when free
    std::vector<long long> len;      // arena length (units) of each slot
    BatchInst* d = nullptr;          // device table
    long long* gstep_d = nullptr;    // device global step counter
    long long gstep = 0;             // host view of the global step
    bool table_dirty = false;        // host copy newer than the device table
    std::vector<int> fresh;          // slots whose Courant maxima must be computed
    int* fresh_d = nullptr;
    // arena
    Arena arena;
    double* arena_mem = nullptr;
    // work lists: [list][dir-1]; list 0 holds the first sweeps of an
    // even-parity step, list 1 the second sweeps; one list per direction, as
    // runs of items (ItemRun, at most one per slot) and their first indices
    ItemRun* runs_d[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int* first_d[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int nruns[2][2] = {{0, 0}, {0, 0}};
    int nitems[2][2] = {{0, 0}, {0, 0}};
    long long lists_step = -1;       // global step the lists' parities refer to
    bool lists_dirty = true;
    unsigned int* counters = nullptr;  // [2 phases][2 directions]
    // graphs for the two step parities
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graphs_dirty = true;
    Tuning tune;
    long long launches = 0;
};

namespace {

long long units_for(const hydroparam_t* H) {
    const long long vs = ((long long)H->nx + 4) * ((long long)H->ny + 4);
    return (4 * vs + 31) / 32;  // one buffer, rounded to 256 bytes
}

int sync_table_down(hb_batch* b) {
    HB_BCU(cudaStreamSynchronize(b->stream));
    if (b->table_dirty) return HB_OK;
    HB_BCU(cudaMemcpy(b->h.data(), b->d, sizeof(BatchInst) * b->capacity, cudaMemcpyDeviceToHost));
    HB_BCU(cudaMemcpy(&b->gstep, b->gstep_d, sizeof(long long), cudaMemcpyDeviceToHost));
    return HB_OK;
}

int sync_table_up(hb_batch* b) {
    if (!b->table_dirty) return HB_OK;
    HB_BCU(cudaMemcpyAsync(b->d, b->h.data(), sizeof(BatchInst) * b->capacity,
                           cudaMemcpyHostToDevice, b->stream));
    HB_BCU(cudaStreamSynchronize(b->stream));
    b->table_dirty = false;
    return HB_OK;
}

// Lists for the current global step: list 0 holds each active instance's
// first-sweep items (x on even nstep, y on odd), list 1 its second-sweep
// items, each split by direction.  One run per instance and list (ItemRun).
int build_lists(hb_batch* b) {
    std::vector<ItemRun> R[2][2];
    std::vector<int> F[2][2];
    long long n[2][2] = {{0, 0}, {0, 0}};
    auto add = [&](int w, int d, const ItemRun& r, long long count) {
        R[w][d].push_back(r);
        F[w][d].push_back((int)n[w][d]);
        n[w][d] += count;
    };
    for (int s = 0; s < b->capacity; s++) {
        const BatchInst& I = b->h[s];
        if (b->off[s] < 0 || !I.active) continue;
        const bool even = (I.nstep % 2) == 0;
        const int xl = even ? 0 : 1, yl = 1 - xl;
        const int groups = (I.nx + hb::kBatchYItemColumns - 1) / hb::kBatchYItemColumns;
        const int segs = (I.ny + b->tune.seg - 1) / b->tune.seg;
        add(yl, 1, ItemRun{s, segs, 0, 0}, (long long)groups * segs);
        // x windows of the stage set's width (two cells per lane in mixed precision)
        const bool mixed = b->precision == HB_PREC_MIXED;
        const int wout = mixed ? hb::kCellWarpOut2 : hb::kCellWarpOut;
        const int nwin = (I.nx + 2 + wout - 1) / wout;
        const int xw = hb::x_item_windows(mixed);
        if (nwin >= xw) {
            const int per = (nwin + xw - 1) / xw;
            add(xl, 0, ItemRun{s, per, nwin, 0}, (long long)I.ny * per);
        } else {
            // A narrow grid: whole rows, as many as make up an item's windows.
            const int rows = xw / nwin;
            add(xl, 0, ItemRun{s, -rows, nwin, 0}, (I.ny + rows - 1) / rows);
        }
    }
    for (int w = 0; w < 2; w++)
        for (int d = 0; d < 2; d++) {
            if (n[w][d] > INT_MAX) return fail(HB_ERR_ARG, "batch: more than 2^31 work items");
            if (!b->runs_d[w][d])
                HB_BCU(cudaMalloc(&b->runs_d[w][d], sizeof(ItemRun) * (size_t)b->capacity));
            if (!b->first_d[w][d])
                HB_BCU(cudaMalloc(&b->first_d[w][d], sizeof(int) * (size_t)b->capacity));
            if (!R[w][d].empty()) {
                HB_BCU(cudaMemcpyAsync(b->runs_d[w][d], R[w][d].data(),
                                       sizeof(ItemRun) * R[w][d].size(), cudaMemcpyHostToDevice,
                                       b->stream));
                HB_BCU(cudaMemcpyAsync(b->first_d[w][d], F[w][d].data(),
                                       sizeof(int) * F[w][d].size(), cudaMemcpyHostToDevice,
                                       b->stream));
            }
            b->nruns[w][d] = (int)R[w][d].size();
            b->nitems[w][d] = (int)n[w][d];
        }
    HB_BCU(cudaStreamSynchronize(b->stream));
    b->lists_step = b->gstep;
    b->lists_dirty = false;
    b->graphs_dirty = true;
    return HB_OK;
}

int grid_size(hb_batch* b, int dir) {
    const int occ = hb::batch_sweep_blocks_per_sm(b->precision == HB_PREC_MIXED,
                                                  b->P.unit_slope != 0, dir, b->tune.threads);
    const int per = (b->tune.blocks_per_sm > 0 && b->tune.blocks_per_sm < occ)
                        ? b->tune.blocks_per_sm
                        : occ;
    return per * b->sm_count;
}

int launch_sweep(hb_batch* b, int list, int phase, cudaStream_t s) {
    for (int dir = 1; dir <= 2; dir++) {
        BatchLaunch L;
        L.inst = b->d;
        L.runs = b->runs_d[list][dir - 1];
        L.run_first = b->first_d[list][dir - 1];
        L.nruns = b->nruns[list][dir - 1];
        L.nitems = b->nitems[list][dir - 1];
        L.phase = phase;
        L.counter = b->counters + 2 * (phase - 1) + (dir - 1);
        L.seg = b->tune.seg;
        L.claim = b->tune.claim;
        L.threads = b->tune.threads;
        if (L.nitems == 0) continue;
        const int grid = grid_size(b, dir);
        HB_BCU(b->precision == HB_PREC_MIXED
                   ? hb::launch_batch_sweep_mixed(L, b->P, dir, grid, s)
                   : hb::launch_batch_sweep(L, b->P, dir, grid, s));
    }
    return HB_OK;
}

// One global step with list parity `flip` (0: lists as built, 1: swapped).
int record_step(hb_batch* b, int flip, cudaStream_t s) {
    HB_BCU(hb::launch_batch_clock_begin(b->d, b->capacity, b->courant_factor, b->P.smallc,
                                        b->gstep_d, s));
    HB_BCU(cudaMemsetAsync(b->counters, 0, 4 * sizeof(unsigned int), s));
    int rc = launch_sweep(b, flip, 1, s);
    if (rc) return rc;
    rc = launch_sweep(b, 1 - flip, 2, s);
    if (rc) return rc;
    HB_BCU(hb::launch_batch_clock_end(b->d, b->capacity, b->gstep_d, s));
    return HB_OK;
}

int build_graphs(hb_batch* b) {
    for (int f = 0; f < 2; f++) {
        if (b->graph[f]) cudaGraphExecDestroy(b->graph[f]);
        b->graph[f] = nullptr;
        cudaGraph_t g = nullptr;
        HB_BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = record_step(b, f, b->stream);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(HB_ERR_CUDA, "end capture", e);
        e = cudaGraphInstantiate(&b->graph[f], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(HB_ERR_CUDA, "graph instantiate", e);
    }
    b->graphs_dirty = false;
    return HB_OK;
}

int prepare(hb_batch* b) {
    int rc = sync_table_up(b);
    if (rc) return rc;
    if (!b->fresh.empty()) {
        HB_BCU(cudaMemcpyAsync(b->fresh_d, b->fresh.data(), sizeof(int) * b->fresh.size(),
                               cudaMemcpyHostToDevice, b->stream));
        HB_BCU(hb::launch_batch_courant(b->d, b->fresh_d, (int)b->fresh.size(), b->P,
                                        b->precision == HB_PREC_MIXED, b->stream));
        b->launches += 1;
        b->fresh.clear();
    }
    if (b->lists_dirty) {
        // The lists follow each instance's step parity: read the clocks first.
        rc = sync_table_down(b);
        if (rc) return rc;
        rc = build_lists(b);
        if (rc) return rc;
    }
    if (b->graphs_dirty) {
        rc = build_graphs(b);
        if (rc) return rc;
    }
    return HB_OK;
}

std::string signature(hb_batch* b) {
    std::vector<std::pair<int, int>> shapes;
    for (int s = 0; s < b->capacity; s++)
        if (b->off[s] >= 0 && b->h[s].active)
            shapes.emplace_back((b->h[s].nx + 63) / 64, (b->h[s].ny + 63) / 64);
    std::sort(shapes.begin(), shapes.end());
    std::string k = std::to_string(b->precision) + ":";
    for (auto& p : shapes) k += std::to_string(p.first) + "x" + std::to_string(p.second) + ",";
    return k;
}

}  // namespace

extern "C" hb_batch* hydro_b200_batch_create(const hydroparam_t* H, int capacity,
                                             size_t arena_bytes, int precision) {
    if (!H || capacity <= 0 || arena_bytes < 256) {
        fail(HB_ERR_ARG, "create: need parameters, capacity > 0 and an arena");
        return nullptr;
    }
    if (precision != HB_PREC_FP64 && precision != HB_PREC_MIXED) {
        fail(HB_ERR_ARG, "create: unknown precision");
        return nullptr;
    }
    if (H->nvar != 4 || H->scheme < 1 || H->scheme > 3 || H->niter_riemann < 0) {
        fail(HB_ERR_ARG, "create: unsupported parameter set");
        return nullptr;
    }
    hb_batch* b = new hb_batch();
    b->capacity = capacity;
    b->precision = precision;
    hb::Phys& P = b->P;
    P.gamma = H->gamma;
    P.gm1 = H->gamma - 1.0;
    P.smallr = H->smallr;
    P.smallc = H->smallc;
    P.smallp = (H->smallc * H->smallc) / H->gamma;
    P.gamma6 = (H->gamma + 1.0) / (2.0 * H->gamma);
    P.smallpp = H->smallr * P.smallp;
    P.entho = 1.0 / (H->gamma - 1.0);
    P.slope_type = H->slope_type;
    P.dx = H->dx;
    P.niter = H->niter_riemann;
    P.iorder = H->iorder;
    P.scheme = H->scheme;
    P.unit_slope = (H->slope_type == 1.0) ? 1 : 0;
    b->courant_factor = H->courant_factor;
    b->h.assign(capacity, BatchInst{});
    b->off.assign(capacity, -1);
    b->len.assign(capacity, 0);
    auto bad = [&](cudaError_t e, const char* what) {
        fail(e == cudaErrorMemoryAllocation ? HB_ERR_NOMEM : HB_ERR_CUDA, what, e);
        hydro_b200_batch_destroy(b);
        return (hb_batch*)nullptr;
    };
    cudaError_t e;
    if ((e = cudaGetDevice(&b->device)) != cudaSuccess) return bad(e, "device");
    if ((e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device)) !=
        cudaSuccess)
        return bad(e, "device attribute");
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bad(e, "stream");
    if ((e = cudaMalloc(&b->d, sizeof(BatchInst) * capacity)) != cudaSuccess)
        return bad(e, "slot table");
    if ((e = cudaMalloc(&b->gstep_d, sizeof(long long))) != cudaSuccess) return bad(e, "counter");
    if ((e = cudaMalloc(&b->counters, 4 * sizeof(unsigned int))) != cudaSuccess)
        return bad(e, "counters");
    if ((e = cudaMalloc(&b->fresh_d, sizeof(int) * capacity)) != cudaSuccess)
        return bad(e, "fresh list");
    if ((e = cudaMalloc(&b->arena_mem, arena_bytes)) != cudaSuccess) return bad(e, "arena");
    b->arena.init(b->arena_mem, (long long)(arena_bytes / 256));
    cudaMemset(b->gstep_d, 0, sizeof(long long));
    b->table_dirty = true;
    if (sync_table_up(b) != HB_OK) {
        hydro_b200_batch_destroy(b);
        return nullptr;
    }
    return b;
}

extern "C" void hydro_b200_batch_destroy(hb_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (int f = 0; f < 2; f++)
        if (b->graph[f]) cudaGraphExecDestroy(b->graph[f]);
    for (int w = 0; w < 2; w++)
        for (int d = 0; d < 2; d++) {
            cudaFree(b->runs_d[w][d]);
            cudaFree(b->first_d[w][d]);
        }
    cudaFree(b->d);
    cudaFree(b->gstep_d);
    cudaFree(b->counters);
    cudaFree(b->fresh_d);
    cudaFree(b->arena_mem);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

extern "C" void* hydro_b200_batch_stream(hb_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" long long hydro_b200_batch_arena_free(hb_batch* b) {
    return b ? b->arena.free_units() * 256 : 0;
}

extern "C" long long hydro_b200_batch_bytes_needed(const hydroparam_t* H) {
    if (!H || H->nx < 3 || H->ny < 3 ||
        ((long long)H->nx + 4) * ((long long)H->ny + 4) > (1ll << 31))
        return 0;  // not an admissible grid
    return 2 * units_for(H) * 256;
}

// Admit an instance: its grid (nx, ny, dx, boundary types) from H, its state
// from host memory (reference layout), clock from t = H->t, nstep = H->nstep.
// Returns the slot, or -1 (no free slot or arena space: HB_ERR_NOMEM).
static int batch_add_impl(hb_batch* b, const hydroparam_t* H, const double* host, double tend,
                          int nstepmax, double dt0);

extern "C" int hydro_b200_batch_add(hb_batch* b, const hydroparam_t* H, const double* host,
                                    double tend, int nstepmax) {
    return batch_add_impl(b, H, host, tend, nstepmax, 0.0);
}

// Resume a checkpointed instance: state from host memory, clock from
// (H->t, H->nstep) and the dt of its last even step (needed when nstep is
// odd: main.c keeps dt for the odd step that follows an even one).
extern "C" int hydro_b200_batch_add_resume(hb_batch* b, const hydroparam_t* H, const double* host,
                                           double dt, double tend, int nstepmax) {
    return batch_add_impl(b, H, host, tend, nstepmax, dt);
}

static int batch_add_impl(hb_batch* b, const hydroparam_t* H, const double* host, double tend,
                          int nstepmax, double dt0) {
    if (!b || !H || !host) return fail(HB_ERR_ARG, "add: null argument"), -1;
    if (H->nx < 3 || H->ny < 3 || !(H->dx > 0.0) ||
        ((long long)H->nx + 4) * ((long long)H->ny + 4) > (1ll << 31))
        return fail(HB_ERR_ARG, "add: unsupported grid"), -1;
    if (sync_table_down(b) != HB_OK) return -1;
    int slot = -1;
    for (int s = 0; s < b->capacity; s++)
        if (b->off[s] < 0) {
            slot = s;
            break;
        }
    if (slot < 0) return fail(HB_ERR_NOMEM, "add: no free slot"), -1;
    const long long u = units_for(H);
    const long long o = b->arena.alloc(2 * u);
    if (o < 0) return fail(HB_ERR_NOMEM, "add: arena full"), -1;
    BatchInst I;
    memset(&I, 0, sizeof(I));
    I.A = b->arena.base + o * 32;
    I.B = I.A + u * 32;
    I.nx = H->nx;
    I.ny = H->ny;
    I.nxt = H->nx + 4;
    I.nyt = H->ny + 4;
    I.vs = (long long)I.nxt * I.nyt;
    I.bnd_left = H->boundary_left;
    I.bnd_right = H->boundary_right;
    I.bnd_down = H->boundary_down;
    I.bnd_up = H->boundary_up;
    I.dx = H->dx;
    I.t = H->t;
    I.dt = dt0;
    I.tend = tend;
    I.nstep = H->nstep;
    I.nstepmax = nstepmax;
    I.active = 1;
    I.stop_step = -1;
    HB_BCU(cudaMemcpyAsync(I.A, host, sizeof(double) * 4 * I.vs, cudaMemcpyHostToDevice,
                           b->stream));
    b->h[slot] = I;
    b->off[slot] = o;
    b->len[slot] = 2 * u;
    b->table_dirty = true;
    b->lists_dirty = true;
    if (I.nstep % 2 == 0) b->fresh.push_back(slot);
    return slot;
}

// Admit an instance whose initial state is a single blast written on the
// device (no host state): density rho, energy e_bg, and e_blast in the
// padded cell (bi, bj).
extern "C" int hydro_b200_batch_add_blast(hb_batch* b, const hydroparam_t* H, double rho,
                                          double e_bg, int bi, int bj, double e_blast, double tend,
                                          int nstepmax) {
    if (!b || !H) return fail(HB_ERR_ARG, "add_blast: null argument"), -1;
    if (H->nx < 3 || H->ny < 3 || bi < 2 || bi >= H->nx + 2 || bj < 2 || bj >= H->ny + 2)
        return fail(HB_ERR_ARG, "add_blast: blast cell outside the interior"), -1;
    if (sync_table_down(b) != HB_OK) return -1;
    int slot = -1;
    for (int s = 0; s < b->capacity; s++)
        if (b->off[s] < 0) {
            slot = s;
            break;
        }
    if (slot < 0) return fail(HB_ERR_NOMEM, "add: no free slot"), -1;
    const long long u = units_for(H);
    const long long o = b->arena.alloc(2 * u);
    if (o < 0) return fail(HB_ERR_NOMEM, "add: arena full"), -1;
    BatchInst I;
    memset(&I, 0, sizeof(I));
    I.A = b->arena.base + o * 32;
    I.B = I.A + u * 32;
    I.nx = H->nx;
    I.ny = H->ny;
    I.nxt = H->nx + 4;
    I.nyt = H->ny + 4;
    I.vs = (long long)I.nxt * I.nyt;
    I.bnd_left = H->boundary_left;
    I.bnd_right = H->boundary_right;
    I.bnd_down = H->boundary_down;
    I.bnd_up = H->boundary_up;
    I.dx = H->dx;
    I.t = H->t;
    I.tend = tend;
    I.nstep = H->nstep;
    I.nstepmax = nstepmax;
    I.active = 1;
    I.stop_step = -1;
    HB_BCU(hb::launch_blast_init(I.A, H->nx, H->ny, rho, e_bg, bi, bj, e_blast, b->stream));
    b->launches += 1;
    b->h[slot] = I;
    b->off[slot] = o;
    b->len[slot] = 2 * u;
    b->table_dirty = true;
    b->lists_dirty = true;
    if (I.nstep % 2 == 0) b->fresh.push_back(slot);
    return slot;
}

extern "C" int hydro_b200_batch_remove(hb_batch* b, int slot) {
    if (!b || slot < 0 || slot >= b->capacity || b->off[slot] < 0)
        return fail(HB_ERR_ARG, "remove: no such slot");
    int rc = sync_table_down(b);
    if (rc) return rc;
    b->arena.release(b->off[slot], b->len[slot]);
    b->off[slot] = -1;
    b->len[slot] = 0;
    memset(&b->h[slot], 0, sizeof(BatchInst));
    b->fresh.erase(std::remove(b->fresh.begin(), b->fresh.end(), slot), b->fresh.end());
    b->table_dirty = true;
    b->lists_dirty = true;
    return HB_OK;
}

// Launch n global steps (asynchronous; one graph launch per step).
extern "C" int hydro_b200_batch_steps(hb_batch* b, int n) {
    if (!b) return fail(HB_ERR_ARG, "steps: null batch");
    int rc = prepare(b);
    if (rc) return rc;
    for (int i = 0; i < n; i++) {
        const int flip = (int)((b->gstep - b->lists_step) & 1);
        HB_BCU(cudaGraphLaunch(b->graph[flip], b->stream));
        b->gstep++;
        b->launches += 6;
    }
    return HB_OK;
}

extern "C" int hydro_b200_batch_synchronize(hb_batch* b) {
    if (!b) return fail(HB_ERR_ARG, "null batch");
    HB_BCU(cudaStreamSynchronize(b->stream));
    return HB_OK;
}

extern "C" int hydro_b200_batch_status(hb_batch* b, int slot, double* t, int* nstep, double* dt,
                                       int* active, long long* stop_step) {
    if (!b || slot < 0 || slot >= b->capacity || b->off[slot] < 0)
        return fail(HB_ERR_ARG, "status: no such slot");
    int rc = sync_table_down(b);
    if (rc) return rc;
    const BatchInst& I = b->h[slot];
    if (t) *t = I.t;
    if (nstep) *nstep = I.nstep;
    if (dt) *dt = I.dt;
    if (active) *active = I.active;
    if (stop_step) *stop_step = I.stop_step;
    return HB_OK;
}

// Activity flags of every slot (1 running, 0 stopped or free) in one read.
extern "C" int hydro_b200_batch_poll(hb_batch* b, int* active, int n) {
    if (!b || !active) return fail(HB_ERR_ARG, "poll: null argument");
    int rc = sync_table_down(b);
    if (rc) return rc;
    for (int s = 0; s < n && s < b->capacity; s++) active[s] = b->off[s] >= 0 && b->h[s].active;
    return HB_OK;
}

// Clocks of the first n slots in one read: active (1 running; 0 stopped or
// free), nstep and t.
extern "C" int hydro_b200_batch_table(hb_batch* b, int* active, int* nstep, double* t, int n) {
    if (!b) return fail(HB_ERR_ARG, "table: null batch");
    int rc = sync_table_down(b);
    if (rc) return rc;
    for (int s = 0; s < n && s < b->capacity; s++) {
        const bool used = b->off[s] >= 0;
        if (active) active[s] = used && b->h[s].active;
        if (nstep) nstep[s] = used ? b->h[s].nstep : 0;
        if (t) t[s] = used ? b->h[s].t : 0.0;
    }
    return HB_OK;
}

extern "C" int hydro_b200_batch_download(hb_batch* b, int slot, double* host) {
    if (!b || !host || slot < 0 || slot >= b->capacity || b->off[slot] < 0)
        return fail(HB_ERR_ARG, "download: no such slot");
    const BatchInst& I = b->h[slot];
    HB_BCU(cudaMemcpyAsync(host, I.A, sizeof(double) * 4 * I.vs, cudaMemcpyDeviceToHost,
                           b->stream));
    HB_BCU(cudaStreamSynchronize(b->stream));
    return HB_OK;
}

extern "C" long long hydro_b200_batch_global_step(hb_batch* b) { return b ? b->gstep : -1; }
extern "C" long long hydro_b200_batch_launch_count(hb_batch* b) { return b ? b->launches : 0; }

extern "C" int hydro_b200_batch_set_tuning(hb_batch* b, int seg, int claim, int blocks_per_sm,
                                           int threads) {
    if (!b || seg < 8 || claim < 1 || blocks_per_sm < 0 || (threads != 64 && threads != 128))
        return fail(HB_ERR_ARG, "set_tuning: invalid values");
    b->tune.seg = seg;
    b->tune.claim = claim;
    b->tune.blocks_per_sm = blocks_per_sm;
    b->tune.threads = threads;
    b->lists_dirty = true;
    b->graphs_dirty = true;
    return HB_OK;
}

extern "C" int hydro_b200_batch_get_tuning(hb_batch* b, int* seg, int* claim,
                                           int* blocks_per_sm, int* threads) {
    if (!b) return fail(HB_ERR_ARG, "get_tuning: null batch");
    if (seg) *seg = b->tune.seg;
    if (claim) *claim = b->tune.claim;
    if (blocks_per_sm) *blocks_per_sm = b->tune.blocks_per_sm;
    if (threads) *threads = b->tune.threads;
    return HB_OK;
}

// Tile autotuner: times `steps` real global steps per candidate tiling --
// threads per CTA (64, 128), y-segment length, items per claim, CTAs per SM
// -- (the tiling does not change any result, so the steps are not wasted) and keeps
// the fastest; remembered per shape signature for later batches.  Returns the
// number of global steps it advanced.
extern "C" int hydro_b200_batch_autotune(hb_batch* b, int steps) {
    if (!b || steps < 1) return fail(HB_ERR_ARG, "autotune: invalid arguments"), -1;
    if (sync_table_down(b) != HB_OK) return -1;
    const std::string key = signature(b);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            b->tune = it->second;
            b->lists_dirty = b->graphs_dirty = true;
            return 0;
        }
    }
    static const int segs[] = {32, 64, 128};
    static const int claims[] = {1, 4, 16};
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return fail(HB_ERR_CUDA, "autotune events"), -1;
    Tuning best = b->tune;
    float best_ms = 1e30f;
    int advanced = 0;
    for (int th : hb::kBatchThreadChoices) {
        const int occ = hb::batch_sweep_blocks_per_sm(b->precision == HB_PREC_MIXED,
                                                      b->P.unit_slope != 0, 2, th);
        const int bpsms[] = {0, std::max(1, occ / 2)};
        for (int sg : segs)
            for (int cl : claims)
                for (int bp : bpsms) {
                    b->tune = Tuning{sg, cl, bp, th};
                    b->lists_dirty = b->graphs_dirty = true;
                    if (prepare(b) != HB_OK) return -1;
                    cudaEventRecord(e0, b->stream);
                    if (hydro_b200_batch_steps(b, steps) != HB_OK) return -1;
                    cudaEventRecord(e1, b->stream);
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    advanced += steps;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = b->tune;
                    }
                }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tune = best;
    b->lists_dirty = b->graphs_dirty = true;
    if (sync_table_down(b) != HB_OK) return -1;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = best;
    }
    return advanced;
}
