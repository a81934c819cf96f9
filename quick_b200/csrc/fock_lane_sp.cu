// The per-lane kernels of the six s/p classes (ssss, psss, psps, ppss, ppps, pppp),
// single-molecule and batched, FP64 and FP32, in a translation unit of their own.
//
// nvcc's code for these straight-line kernels depends on how their compilation unit
// is split for parallel optimisation (--split-compile), and a split compile is not
// deterministic: two compiles of the same unit with the same flags give different
// device code.  Inside the whole library (split over all host cores) psss took
// 2.07-2.36 ms and ssss 1.27-1.49 ms per build of 32 H2O / 6-31G*, from build to
// build.  Compiled alone and without a split (quick_b200/build.py) they get the
// same code on every build: ssss 1.28-1.29 ms, psss 2.07-2.09 ms (timed side by
// side on one GPU).  get2e.cu declares these instantiations extern when the build
// defines QK_LANE_SP_TU_SEPARATE.
#define QK_LANE_SP_TU 1
#include "get2e.cu"

namespace qk {
#if QK_MAX_L >= 1
#define QK_LANE_SP_INST(a, b, c, e)                                                                        \
    template __global__ void fock_class_kernel<a, b, c, e, false>(DevData, const int4*, int, int*);        \
    template __global__ void fock_class_kernel<a, b, c, e, true>(DevData, const int4*, int, int*);         \
    template __global__ void fock_class_kernel_batch<a, b, c, e, false>(const DevData*, const BatchSeg*, int, \
                                                                        int, int*);                          \
    template __global__ void fock_class_kernel_batch<a, b, c, e, true>(const DevData*, const BatchSeg*, int,  \
                                                                       int, int*);
QK_LANE_SP_CLASSES(QK_LANE_SP_INST)
#undef QK_LANE_SP_INST
#endif
}  // namespace qk
