// fftb_fused3d.cu -- specialised fused 3D kernels.
#include "../../include/fftb.h"
#include "fftb_fused3d.h"

namespace fftb {

int fused3d_init(Fused3D &f, int dtype, long long nx, long long ny, long long nz)
{
    f.enabled = false;
    f.dtype = dtype;
    f.nx = nx;
    f.ny = ny;
    f.nz = nz;
    return FFTB_SUCCESS;
}

int fused3d_forward(const Fused3D &, const void *, void *, cudaStream_t, LaunchTimer *)
{
    return FFTB_ERROR_UNSUPPORTED_SIZE;
}
int fused3d_backward(const Fused3D &, void *, void *, double, cudaStream_t, LaunchTimer *)
{
    return FFTB_ERROR_UNSUPPORTED_SIZE;
}
int fused3d_spectral(const Fused3D &, const void *, void *, void *, const EpValues &, cudaStream_t, LaunchTimer *)
{
    return FFTB_ERROR_UNSUPPORTED_SIZE;
}
int fused3d_num_launches(const Fused3D &, int) { return 0; }

} // namespace fftb
