// The single-frame FP64 camera kernel of the plain path (the fast path computes the same in its
// batch kernel); the computation itself is in sr_camera.cuh.
#include "sr_camera.cuh"
#include "sr_kernels.h"

namespace srk {

__global__ void k_camera_f64(SrCameraF64 c, double a0, double a1, double a2, double a3, SrGpuUniforms U, float4* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double anchor[4] = {a0, a1, a2, a3};
    camera_f64(c, anchor, U, out);
}

cudaError_t launch_camera_f64(const SrCameraF64& c, const double anchor[4], const SrGpuUniforms& u, float4* cam_dev,
                              cudaStream_t st) {
    k_camera_f64<<<1, 32, 0, st>>>(c, anchor[0], anchor[1], anchor[2], anchor[3], u, cam_dev);
    return cudaGetLastError();
}

}  // namespace srk
