// fftb_fused3d.h -- specialised 3D kernels (fused multi-axis passes) for the
// sizes that have them; the generic pass programs cover every other size.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "fftb_engine.h"

namespace fftb {

struct Fused3D {
    bool enabled = false;
    int dtype = 0;
    long long nx = 0, ny = 0, nz = 0;
    int cluster = 0;               // CTAs per (y, z) plane of the forward plane kernel
    int cluster_inv = 0;           // the same for the inverse plane kernel (may differ)
    bool tc = false;               // column kernels with the first radix-16 stage on the tensor cores
    const void *plane = nullptr;   // selected plane kernel entry (forward)
    const void *plane_inv = nullptr;  // entry whose inverse kernel runs (its own cluster size)
    const void *xcol = nullptr;    // selected x column kernel entry
    void *roots_plane = nullptr;   // device root table of length max(ny, nz)
    void *roots_x = nullptr;       // device root table of length nx
};

// Sets f.enabled when (dtype, nx, ny, nz) has a specialised path.  force_cluster = 0
// picks the plane cluster size by occupancy; 1, 2, 4 or 8 asks for that size (f stays
// disabled when the size has no such plane kernel).
int fused3d_init(Fused3D &f, int dtype, long long nx, long long ny, long long nz, int force_cluster = 0);
// The cluster sizes with plane kernels for (dtype, ny, nz) that fit the shared memory of a CTA.
int fused3d_clusters(int dtype, long long nx, long long ny, long long nz, int *clusters, int cap);
int fused3d_forward(const Fused3D &f, const void *in, void *out, cudaStream_t s, LaunchTimer *t);
int fused3d_backward(const Fused3D &f, void *in, void *out, double scale, cudaStream_t s, LaunchTimer *t);
int fused3d_spectral(const Fused3D &f, const void *in, void *out, void *work, const EpValues &ep, cudaStream_t s,
                     LaunchTimer *t);
int fused3d_forward_adjoint(const Fused3D &f, void *gspec, void *greal, cudaStream_t s, LaunchTimer *t);
int fused3d_backward_adjoint(const Fused3D &f, const void *greal, void *gspec, cudaStream_t s, LaunchTimer *t);
// du/d(axis) (0 = x, 1 = y, 2 = z) through the spectrum buffer spec: 3 launches
int fused3d_derivative(const Fused3D &f, const void *in, void *spec, void *out, int axis, cudaStream_t s,
                       LaunchTimer *t);
// all three first derivatives: 7 launches, the spectrum written once and read per axis
int fused3d_gradient(const Fused3D &f, const void *in, void *spec, void *spec2, void *const *outs, cudaStream_t s,
                     LaunchTimer *t);
int fused3d_num_launches(const Fused3D &f, int which);

// The x or y FFTs of many f32 3D spectra [nx][ny][nz/2+1] of one line length in one launch,
// one CTA per tile of lines, with the column kernel's register-resident FFT (the batched
// transforms' column stages).  kind: 0 x forward, 1 x inverse, 2 x sandwich (forward,
// spectral multiply, inverse), 3 y forward, 4 y inverse.
struct XGroupItem {
    long long off;  // complex elements from the buffer base to the spectrum
    int ncols;      // lines of the spectrum: x kinds ny * (nz/2 + 1), y kinds nx * (nz/2 + 1)
    int tile;       // tile of col_group_tile_lines(n) lines
    int ny, nz;
};
// 0 when no grouped column kernel exists for this line length, else the lines per tile
int col_group_tile_lines(int dtype, int n);
// Raises the kernel's shared-memory limit and returns the root table of length n.
int col_group_prepare(int dtype, int kind, int n, void **roots);
// ep_mode / scale / sign: the sandwich's multiply (EP_SCALE, EP_POISSON as the pass epilogue)
int launch_col_group(int kind, int n, const XGroupItem *items, int nitems, void *data, const void *roots,
                     int ep_mode, double scale, double sign, cudaStream_t s);

// The z stage of many f32 3D transforms of one z length (32-256, a power of two) in one launch:
// R2C (dir 0) or scaled C2R (dir 1) of two contiguous real rows per complex FFT.
struct RowGroupItem {
    long long roff;  // floats from the real buffer base to the transform's rows [nrows][nz]
    long long soff;  // complex elements from the spectrum buffer base to its rows [nrows][nz/2+1]
    int nrows;       // rows (nx * ny)
    int tile;        // tile of row_group_tile_pairs(nz) row pairs
    float scale;     // C2R output scale
};
int row_group_tile_pairs(int dtype, int nz);
// dynamic shared memory of one row-pair tile / one column tile
size_t row_group_smem(int nz);
size_t col_group_smem(int n);
int row_group_prepare(int dtype, int dir, int nz, void **roots);
int launch_row_group(int dir, int nz, const RowGroupItem *items, int nitems, const void *in, void *out,
                     const void *roots, cudaStream_t s);

// 4D slab / native_xzwy with power-of-two (z, w) planes and x, y column kernels.
struct Fused4D {
    bool enabled = false;
    int dtype = 0, layout = 0;
    long long nx = 0, ny = 0, nz = 0, nw = 0;
    bool tc = false;               // column kernels with the first radix-16 stage on the tensor cores
    const void *plane = nullptr, *xcol = nullptr, *ycol = nullptr;
    void *roots_plane = nullptr, *roots_x = nullptr, *roots_y = nullptr;
};
int fused4d_init(Fused4D &f, int dtype, int layout, long long nx, long long ny, long long nz, long long nw);
int fused4d_forward(const Fused4D &f, const void *in, void *out, void *work, cudaStream_t s, LaunchTimer *t);
int fused4d_backward(const Fused4D &f, void *in, void *out, void *work, double scale, cudaStream_t s,
                     LaunchTimer *t);
int fused4d_spectral(const Fused4D &f, const void *in, void *out, void *work, const EpValues &ep, cudaStream_t s,
                     LaunchTimer *t);
int fused4d_forward_adjoint(const Fused4D &f, void *gspec, void *greal, void *work, cudaStream_t s, LaunchTimer *t);
int fused4d_backward_adjoint(const Fused4D &f, const void *greal, void *gspec, void *work, cudaStream_t s,
                             LaunchTimer *t);
int fused4d_num_launches(const Fused4D &f, int which);

} // namespace fftb
