// hb_output.cu -- the reference's VTK output written from the device state.
//
// vtkfile.c:140-306 writes, for each variable, the interior cells converted to
// float (C's (float) cast: round to nearest even), base64-encoded after a
// base64-encoded 4-byte length; plus coordinates, a parallel header (.pvtr)
// and a collection file (Hydro.pvd).  Here the float conversion and the
// base64 encoding run on the GPU over the resident state, so an output step
// moves 5.3 bytes per cell and variable to the host instead of the 32-byte
// cell state, and the host only writes text.  The file layout, names and
// every formatted line follow vtkfile.c, so the files are byte-identical to
// the reference's (tested against the reference application).
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <sys/types.h>

#include "hb_kernels.cuh"
#include "../../include/hydro_b200.h"

int hb_record_error(int code, const char* msg);  // hb_runtime.cu

namespace hb {

// Standard base64 alphabet (RFC 4648 section 4), as vtkfile.c:31-46 maps it.
__device__ __forceinline__ unsigned char b64_char(unsigned int x) {
    return x < 26 ? (unsigned char)('A' + x)
         : x < 52 ? (unsigned char)('a' + (x - 26))
         : x < 62 ? (unsigned char)('0' + (x - 52))
         : x == 62 ? (unsigned char)'+' : (unsigned char)'/';
}

__device__ __forceinline__ float cell_float(const double* __restrict__ u, int m, int nx,
                                            int nxt) {
    const int j = m / nx, i = m - j * nx;
    return __double2float_rn(__ldg(u + (long long)(j + 2) * nxt + (i + 2)));
}

// Thread t encodes floats 3t .. 3t+2 (12 bytes, 4 groups, 16 characters);
// the last thread also handles a tail of 1 or 2 floats with '=' padding
// (vtkfile.c:47-102).
__global__ void vtk_base64_kernel(const double* __restrict__ u, int nx, int ny, int nxt,
                                  unsigned char* __restrict__ out) {
    const int n = nx * ny;
    const int full = n / 3;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nf = t < full ? 3 : (t == full ? n - 3 * full : 0);
    if (nf == 0) return;
    unsigned char b[12];
    for (int f = 0; f < 3; f++) {
        unsigned int w = 0u;
        if (f < nf) w = __float_as_uint(cell_float(u, 3 * t + f, nx, nxt));
        b[4 * f + 0] = (unsigned char)(w & 0xffu);  // little-endian bytes of the float
        b[4 * f + 1] = (unsigned char)((w >> 8) & 0xffu);
        b[4 * f + 2] = (unsigned char)((w >> 16) & 0xffu);
        b[4 * f + 3] = (unsigned char)(w >> 24);
    }
    const int nbytes = 4 * nf;
    unsigned char c[16];
    int nc = 0;
    for (int g = 0; g * 3 < nbytes; g++) {
        const int left = nbytes - 3 * g;  // bytes of this group present
        const unsigned int b1 = b[3 * g], b2 = left > 1 ? b[3 * g + 1] : 0u,
                           b3 = left > 2 ? b[3 * g + 2] : 0u;
        c[nc++] = b64_char(b1 >> 2);
        c[nc++] = b64_char(((b1 & 0x03u) << 4) | (b2 >> 4));
        c[nc++] = left > 1 ? b64_char(((b2 & 0x0fu) << 2) | (b3 >> 6)) : (unsigned char)'=';
        c[nc++] = left > 2 ? b64_char(b3 & 0x3fu) : (unsigned char)'=';
    }
    unsigned char* o = out + 16ll * t;
    if (nc == 16) {
        uint4 v;
        memcpy(&v, c, 16);
        *reinterpret_cast<uint4*>(o) = v;  // out is 16-byte aligned, offset 16t
    } else {
        for (int k = 0; k < nc; k++) o[k] = c[k];
    }
}

cudaError_t launch_vtk_base64(const double* var_plane, int nx, int ny, int nxt,
                              unsigned char* out, cudaStream_t s) {
    const int n = nx * ny;
    const int threads = n / 3 + 1;
    vtk_base64_kernel<<<(threads + 255) / 256, 256, 0, s>>>(var_plane, nx, ny, nxt, out);
    return cudaGetLastError();
}

}  // namespace hb

// ---------------------------------------------------------------- the writer

// Length of the base64 text of nbytes bytes (vtkfile.c:48-63).
static long long b64_len(long long nbytes) { return nbytes ? 4 * ((nbytes - 1) / 3 + 1) : 0; }

static std::string b64_host(const unsigned char* data, int len) {
    static const char* A = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::string s;
    for (int i = 0; i < len; i += 3) {
        const unsigned int b1 = data[i], b2 = i + 1 < len ? data[i + 1] : 0u,
                           b3 = i + 2 < len ? data[i + 2] : 0u;
        s += A[b1 >> 2];
        s += A[((b1 & 3u) << 4) | (b2 >> 4)];
        s += i + 1 < len ? A[((b2 & 15u) << 2) | (b3 >> 6)] : '=';
        s += i + 2 < len ? A[b3 & 63u] : '=';
    }
    return s;
}

extern "C" long long hydro_b200_vtk_base64_len(int nx, int ny) {
    if (nx <= 0 || ny <= 0) return 0;
    return b64_len(4ll * nx * ny);
}

// Boxes of the simple decomposition (SplitSurface.c:102-185), for the piece
// list of the parallel header when the run is split over nproc ranks.
static void sub_surface(int gx, int gy, int nproc, int me, int box[4]) {
    int py = (int)sqrt((double)nproc);
    int res = (nproc - py * py) / py;
    int px = py + res;
    if (px * py != nproc) {
        int divider = 2, last = 1;
        while (divider < (int)sqrt((double)nproc)) {
            if (nproc % divider == 0) last = divider;
            divider++;
        }
        py = last;
        res = (nproc - py * py) / py;
        px = py + res;
    }
    const int pex = me % px, pey = me / px;
    int incx = (gx + 1) / px, incy = (gy + 1) / py;
    if (incx * px < gx) incx++;
    if (incy * py < gy) incy++;
    box[0] = pex * incx < 0 ? 0 : pex * incx;
    box[1] = (pex + 1) * incx > gx ? gx : (pex + 1) * incx;
    box[2] = pey * incy < 0 ? 0 : pey * incy;
    box[3] = (pey + 1) * incy > gy ? gy : (pey + 1) * incy;
}

static int make_dir(const char* p) {
    if (mkdir(p, 0777) == 0 || errno == EEXIST) return 0;
    return -1;
}

// vtkfile.c:109-127 (Hydro.pvd listing every output so far).
static int write_pvd(int nout) {
    FILE* vf = fopen("Hydro.pvd", "w");
    if (!vf) return -1;
    fprintf(vf, "<?xml version=\"1.0\"?>\n");
    fprintf(vf, " <VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    fprintf(vf, "  <Collection>\n");
    for (int i = 1; i <= nout; i++) {
        char tmp[32];
        snprintf(tmp, sizeof(tmp), "%06d", i);
        fprintf(vf, "  <DataSet timestep=\"%d\" part=\"0\" file=\"Dep/%.4s/%.2s/Hydro_%04d.pvtr\"  "
                    "name=\"Asmb:FRAME\"/>\n",
                i, tmp, tmp + 4, i);
    }
    fprintf(vf, " </Collection>\n");
    fprintf(vf, "</VTKFile>\n");
    return fclose(vf);
}

int hb_vtk_write(hb_domain* d, int step, const hydroparam_t* H) {
    static const char* kNames[4] = {"varID", "varIU", "varIV", "varIP"};
    // Dep/XXXX/YY for output number `step` (vtkfile.c:129-148); every rank
    // creates it, mkdir tolerating an existing directory.
    char tmp[32], dir[64], name[160];
    snprintf(tmp, sizeof(tmp), "%06d", step);
    snprintf(dir, sizeof(dir), "Dep");
    if (make_dir(dir)) return hb_record_error(HB_ERR_ARG, "vtkfile: cannot create Dep");
    snprintf(dir, sizeof(dir), "Dep/%.4s", tmp);
    if (make_dir(dir)) return hb_record_error(HB_ERR_ARG, "vtkfile: cannot create directory");
    snprintf(dir, sizeof(dir), "Dep/%.4s/%.2s", tmp, tmp + 4);
    if (make_dir(dir)) return hb_record_error(HB_ERR_ARG, "vtkfile: cannot create directory");

    const long long nb = hydro_b200_vtk_base64_len(H->nx, H->ny);
    std::vector<char> text((size_t)nb + 16);
    snprintf(name, sizeof(name), "%s/Hydro_%05d_%04d.vtr", dir, H->mype, step);
    FILE* fic = fopen(name, "w");
    if (!fic) return hb_record_error(HB_ERR_ARG, "vtkfile: cannot open the piece file");
    const int* box = H->box;
    fprintf(fic, "<?xml version=\"1.0\"?>\n");
    fprintf(fic, "<VTKFile type=\"RectilinearGrid\" byte_order=\"LittleEndian\">\n");
    fprintf(fic, " <RectilinearGrid WholeExtent=\" %d %d %d %d %d %d\">\n", box[0], box[1],
            box[2], box[3], 0, 1);
    fprintf(fic, "  <Piece Extent=\" %d %d %d %d %d %d\" GhostLevel=\"0\">\n", box[0], box[1],
            box[2], box[3], 0, 1);
    fprintf(fic, "   <Coordinates>\n");
    fprintf(fic, "    <DataArray type=\"Float32\" format=\"ascii\" NumberOfComponents=\"1\">\n");
    for (int i = box[0]; i <= box[1]; i++) fprintf(fic, "%f ", i * H->dx);
    fprintf(fic, "\n");
    fprintf(fic, "    </DataArray>\n");
    fprintf(fic, "    <DataArray type=\"Float32\" format=\"ascii\" NumberOfComponents=\"1\">\n");
    for (int j = box[2]; j <= box[3]; j++) fprintf(fic, "%f ", j * H->dx);
    fprintf(fic, "\n");
    fprintf(fic, "    </DataArray>\n");
    fprintf(fic, "    <DataArray type=\"Float32\" format=\"ascii\" NumberOfComponents=\"1\">\n");
    fprintf(fic, "%f %f\n", 0., 1. * H->dx);
    fprintf(fic, "    </DataArray>\n");
    fprintf(fic, "   </Coordinates>\n");
    fprintf(fic, "   <CellData Scalars=\" varID varIU varIV varIP\">\n");
    // The length header: base64 of the first 4 bytes of the byte count
    // (vtkfile.c:271-276; little-endian).
    const unsigned int payload = (unsigned int)(4ull * H->nx * H->ny);
    unsigned char hdr[4] = {(unsigned char)(payload & 0xff), (unsigned char)((payload >> 8) & 0xff),
                            (unsigned char)((payload >> 16) & 0xff),
                            (unsigned char)(payload >> 24)};
    const std::string h64 = b64_host(hdr, 4);
    int rc = HB_OK;
    for (int nv = 0; nv < 4 && rc == HB_OK; nv++) {
        fprintf(fic,
                "    <DataArray Name=\"%s\" type=\"Float32\" format=\"binary\" encoding=\"base64\" "
                "NumberOfComponents=\"1\">\n",
                kNames[nv]);
        rc = hydro_b200_domain_vtk_base64(d, nv, text.data(), nb);
        if (rc != HB_OK) break;
        fwrite(h64.data(), 1, h64.size(), fic);
        fwrite(text.data(), 1, (size_t)nb, fic);
        fprintf(fic, "    </DataArray>\n");
    }
    fprintf(fic, "   </CellData>\n");
    fprintf(fic, "  </Piece>\n");
    fprintf(fic, " </RectilinearGrid>\n");
    fprintf(fic, "</VTKFile>\n");
    if (fclose(fic) != 0 && rc == HB_OK) rc = hb_record_error(HB_ERR_ARG, "vtkfile: write failed");
    if (rc != HB_OK || H->mype != 0) return rc;

    // Parallel header and collection, rank 0 only (vtkfile.c:286-349).
    snprintf(name, sizeof(name), "%s/Hydro_%04d.pvtr", dir, step);
    FILE* vf = fopen(name, "w");
    if (!vf) return hb_record_error(HB_ERR_ARG, "vtkfile: cannot open the parallel header");
    fprintf(vf, "<?xml version=\"1.0\"?>\n");
    fprintf(vf, "<VTKFile type=\"PRectilinearGrid\" byte_order=\"LittleEndian\">\n");
    fprintf(vf, "<PRectilinearGrid WholeExtent=\"0 %d 0 %d 0 %d\"  GhostLevel=\"0\" >\n",
            H->globnx, H->globny, 1);
    fprintf(vf, " <PCellData>\n");
    for (int nv = 0; nv < 4; nv++)
        fprintf(vf,
                "  <PDataArray Name=\"%s\" type=\"Float32\" format=\"binary\" "
                "encoding=\"base64\" NumberOfComponents=\"1\"/>\n",
                kNames[nv]);
    fprintf(vf, " </PCellData>\n");
    fprintf(vf, " <PCoordinates>\n");
    for (int k = 0; k < 3; k++)
        fprintf(vf, "  <PDataArray type=\"Float32\" format=\"ascii\" NumberOfComponents=\"1\"/>\n");
    fprintf(vf, " </PCoordinates>\n");
    for (int r = 0; r < H->nproc; r++) {
        int b[4] = {0, H->globnx, 0, H->globny};
        if (H->nproc > 1) sub_surface(H->globnx, H->globny, H->nproc, r, b);
        fprintf(vf, " <Piece Extent=\"%d %d %d %d %d %d\" Source=\"Hydro_%05d_%04d.vtr\"/>\n", b[0],
                b[1], b[2], b[3], 0, 1, r, step);
    }
    fprintf(vf, "</PRectilinearGrid>\n");
    fprintf(vf, "</VTKFile>\n");
    if (fclose(vf) != 0) return hb_record_error(HB_ERR_ARG, "vtkfile: write failed");
    if (write_pvd(step) != 0) return hb_record_error(HB_ERR_ARG, "vtkfile: cannot write Hydro.pvd");
    return HB_OK;
}
