// hb_noalloc.cu -- a time step that allocates no memory.
//
// Some callers cannot call cudaMalloc at all: code that runs inside another
// framework's memory arena (which owns all of the device memory it will give
// out), or inside a process whose device allocations are capped by a budget
// it has already spent.  They still want the fused sweeps, which need one
// scratch buffer the size of the state (the first sweep writes it, the second
// reads it back).  This file provides that scratch as a file-scope __device__
// array of fixed size, so hydro_b200_godunov_noalloc() performs one
// hydro_godunov step on a state the caller already holds on the device,
// calling no cudaMalloc, cudaFree, stream or event creation.  It launches the
// kernels the regular path uses for grids of this size: the x sweep and the
// y sweep with one cell per lane (xcell_kernel, ycell_kernel), so its results
// are bitwise those of hydro_godunov.
//
// Limits and sharing:
//   * the state may hold at most HB_NOALLOC_MAX_CELLS padded cells
//     ((nx+4)*(ny+4)), i.e. the scratch is 4 * 2^20 doubles = 32 MiB, held by
//     every GPU that loads this library until the process exits;
//   * every call uses the same array: calls whose kernels overlap on the GPU
//     (different streams, or different host threads on one device) race on
//     it and must be serialised by the caller.  Nothing in it needs to start
//     at zero -- the first sweep writes every cell the second sweep reads;
//   * the state must be device (or managed) memory of the current device,
//     checked with cudaPointerGetAttributes: a pointer of another device or
//     of host memory is rejected with HB_ERR_ARG instead of being read by
//     kernels that cannot reach it.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/hydro_b200.h"
#include "hb_kernels.cuh"

int hb_record_error(int code, const char* msg);  // hb_runtime.cu

namespace {

constexpr long long kScratchDoubles = 4ll * HB_NOALLOC_MAX_CELLS;

// The scratch buffer (one per device that loads the library).
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// In host code g_noalloc_scratch names a host-side stand-in, not a device
// address: its device address is looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// hydro_godunov's constants with the reference's formulas (the same
// derivation the domain runtime uses).
hb::Phys phys_from(const hydroparam_t* H) {
    hb::Phys P;
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
    return P;
}

hb::SweepArgs args_for(const hydroparam_t* H, int dir, const double* in, double* out,
                       double* state, double dt) {
    hb::SweepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in = in;
    a.resid = state;
    a.out = out;
    a.gout = state;
    a.clk = nullptr;
    a.dt = dt;
    a.courant = nullptr;
    a.nx = H->nx;
    a.ny = H->ny;
    a.nxt = H->nx + 4;
    a.nyt = H->ny + 4;
    a.vs = (long long)a.nxt * a.nyt;
    if (dir == 1) {
        a.bnd_lo = H->boundary_left;
        a.bnd_hi = H->boundary_right;
        a.nlines = H->ny;
        a.n = a.nxt;
    } else {
        a.bnd_lo = H->boundary_down;
        a.bnd_hi = H->boundary_up;
        a.nlines = H->nx;
        a.n = a.nyt;
    }
    a.seg = 0;  // the cell-per-lane kernels take no segment length
    a.w_lo = 0;
    a.w_hi = hb::kWholeLine;
    return a;
}

}  // namespace

extern "C" int hydro_b200_godunov_noalloc(const hydroparam_t* H, double* d_uold, int idim,
                                          double dt, void* stream) {
    if (!H || !d_uold) return hb_record_error(HB_ERR_ARG, "noalloc: null parameters or state");
    if (idim != 1 && idim != 2) return hb_record_error(HB_ERR_ARG, "noalloc: idim must be 1 or 2");
    if (H->nvar != 4 || H->nx < 3 || H->ny < 3 || H->scheme < 1 || H->scheme > 3 ||
        !(H->dx > 0.0) || H->niter_riemann < 0)
        return hb_record_error(HB_ERR_ARG, "noalloc: unsupported parameter set");
    // The state is read with the strides nx+4, ny+4 (as hydro_b200_domain_create
    // requires; 0 leaves them unset, as the reference's reader does until
    // hydro_init).
    if ((H->nxt && H->nxt != H->nx + 4) || (H->nyt && H->nyt != H->ny + 4))
        return hb_record_error(HB_ERR_ARG, "noalloc: nxt/nyt must be nx+4, ny+4");
    if (((long long)H->nx + 4) * ((long long)H->ny + 4) > HB_NOALLOC_MAX_CELLS)
        return hb_record_error(HB_ERR_ARG,
                               "noalloc: grid too large: (nx+4)*(ny+4) must be <= "
                               "HB_NOALLOC_MAX_CELLS (1048576 padded cells, 32 MiB of scratch)");

    // The kernels run on this runtime's current device: the state must live
    // there.  Any failure of the query (a host pointer on a machine without a
    // device included) means the pointer cannot be used.
    cudaPointerAttributes attr;
    std::memset(&attr, 0, sizeof(attr));
    if (cudaPointerGetAttributes(&attr, d_uold) != cudaSuccess) {
        cudaGetLastError();  // the query's error is not sticky; clear it
        return hb_record_error(HB_ERR_ARG, "noalloc: d_uold is not a device pointer");
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return hb_record_error(HB_ERR_CUDA, "noalloc: no usable current device");
    if (!(attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) ||
        attr.device != dev)
        return hb_record_error(HB_ERR_ARG,
                               "noalloc: d_uold must be device or managed memory of the current "
                               "device (see hydro_b200_set_device)");
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_ptr[dev]) {
            // First call on this device: look up the device address of the
            // scratch array (this device is current here).
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
                return hb_record_error(HB_ERR_CUDA, "noalloc: cudaGetSymbolAddress failed");
            g_scratch_ptr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_ptr[dev];
    }

    const hb::Phys P = phys_from(H);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int first = (idim == 1) ? 1 : 2;
    const int second = 3 - first;
    // hydro_godunov.c:70-139: first sweep state -> scratch, second scratch -> state.
    // The FP64 kernels the domain path uses for grids of at most 8 M cells.
    auto launch = [&](int dir, const hb::SweepArgs& a) {
        return dir == 1 ? hb::launch_xcell(a, P, s) : hb::launch_ycell(a, P, s);
    };
    if (launch(first, args_for(H, first, d_uold, scratch, d_uold, dt)) != cudaSuccess)
        return hb_record_error(HB_ERR_CUDA, "noalloc: sweep launch failed");
    if (launch(second, args_for(H, second, scratch, d_uold, d_uold, dt)) != cudaSuccess)
        return hb_record_error(HB_ERR_CUDA, "noalloc: sweep launch failed");
    return HB_OK;
}
