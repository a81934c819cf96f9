// TEST INFRASTRUCTURE ONLY: QUICK's own GPU host code plus one timing hook.
//
// This unit compiles the reference's src/gpu/cuda/gpu.cu from the reference tree
// (found through the include path; nothing of it is copied here) and adds
// refgpu_time_get2e, which launches the reference's Fock-build kernels -- get2e()
// (src/gpu/cuda/gpu_get2e.cu:594-637), exactly what gpu_get_cshell_eri_ launches
// (src/gpu/gpu_get2e_getxc_drivers.h:30-38) -- between two CUDA events on the
// legacy default stream those kernels run on.  gpu.cu keeps its state in a
// file-scope `gpu` object, so the hook must live in the same translation unit.
#include "gpu.cu"

extern "C" int refgpu_time_get2e(int nrep, void* flush, size_t flush_bytes, float* ms) {
    if (!gpu || !gpu->gpu_calculated || !gpu->gpu_calculated->oULL) return 1;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return 2;
    upload_sim_to_constant(gpu);
    const size_t nn = (size_t)gpu->nbasis * gpu->nbasis;
    for (int r = 0; r < nrep; ++r) {
        // every repetition starts from a cleared accumulator and a cold L2
        cudaMemsetAsync(gpu->gpu_calculated->oULL->_devData, 0, sizeof(QUICKULL) * nn, 0);
        if (flush && flush_bytes) cudaMemsetAsync(flush, r & 0xff, flush_bytes, 0);
        cudaEventRecord(e0, 0);
        get2e(gpu);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms[r], e0, e1);
    }
    cudaMemsetAsync(gpu->gpu_calculated->oULL->_devData, 0, sizeof(QUICKULL) * nn, 0);
    cudaError_t e = cudaDeviceSynchronize();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return e == cudaSuccess ? 0 : 3;
}
