// Device helpers of the SCF iteration that must stay on the GPU stream (no host
// synchronisation), so that a whole iteration can be captured as a CUDA graph.
//
// small_solve_kernel: the Pulay DIIS system (QUICK's electdiis,
// src/modules/quick_scf_module.f90:165-802, which solves it on the host with
// LAPACK) -- at most 64 unknowns -- by Gaussian elimination with partial
// pivoting in one warp, the matrix held in shared memory.  A zero or non-finite
// pivot sets *ok = 0 (the caller then keeps the plain Fock matrix).
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

#include "quick_b200.h"

namespace qk {

constexpr int kSmallSolveMax = 64;

__global__ void __launch_bounds__(32) small_solve_kernel(const double* __restrict__ A, const double* __restrict__ b,
                                                         int n, double* __restrict__ x, int* __restrict__ ok) {
    __shared__ double M[kSmallSolveMax][kSmallSolveMax + 1];
    __shared__ int good;
    const int lane = threadIdx.x;
    for (int i = 0; i < n; ++i) {
        for (int j = lane; j < n; j += 32) M[i][j] = A[(size_t)i * n + j];
        if (lane == 0) M[i][n] = b[i];
    }
    if (lane == 0) good = 1;
    __syncwarp();
    for (int k = 0; k < n; ++k) {
        // pivot: largest |M[i][k]|, i >= k (lowest index on ties)
        double best = -1.0;
        int bi = k;
        for (int i = k + lane; i < n; i += 32) {
            const double v = fabs(M[i][k]);
            if (v > best) { best = v; bi = i; }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (!(best > 0.0) || !isfinite(best)) {
            if (lane == 0) good = 0;
            break;
        }
        if (bi != k)
            for (int j = lane; j <= n; j += 32) {
                const double t = M[k][j];
                M[k][j] = M[bi][j];
                M[bi][j] = t;
            }
        __syncwarp();
        const double piv = M[k][k];
        for (int i = k + 1; i < n; ++i) {
            const double f = M[i][k] / piv;
            __syncwarp();
            for (int j = k + lane; j <= n; j += 32) M[i][j] -= f * M[k][j];
            __syncwarp();
        }
    }
    __syncwarp();
    if (lane == 0) {
        if (good) {
            for (int i = n - 1; i >= 0; --i) {
                double s = M[i][n];
                for (int j = i + 1; j < n; ++j) s -= M[i][j] * x[j];
                x[i] = s / M[i][i];
                if (!isfinite(x[i])) good = 0;
            }
        }
        if (!good)
            for (int i = 0; i < n; ++i) x[i] = 0.0;
        *ok = good;
    }
}

// One step of SP2 purification (Niklasson, Phys. Rev. B 66, 155115 (2002)) after
// Y2 = Y Y: Yout = Y2 when |tr Y2 - ne| < |2 tr Y - tr Y2 - ne|, else 2Y - Y2.
// Every block sums both traces itself, in the same fixed order, so all blocks take
// the same branch without a second launch; Yout must not alias Y or Y2.
constexpr int kSp2Threads = 256;

__global__ void __launch_bounds__(kSp2Threads) sp2_step_kernel(const double* __restrict__ Y,
                                                               const double* __restrict__ Y2,
                                                               double* __restrict__ Yout, int n, double ne) {
    __shared__ double part[2][kSp2Threads / 32];
    __shared__ int square;
    double t0 = 0.0, t1 = 0.0;
    for (int i = threadIdx.x; i < n; i += kSp2Threads) {
        t0 += Y[(size_t)i * (n + 1)];
        t1 += Y2[(size_t)i * (n + 1)];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t0 += __shfl_xor_sync(0xffffffffu, t0, o);
        t1 += __shfl_xor_sync(0xffffffffu, t1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part[0][threadIdx.x >> 5] = t0;
        part[1][threadIdx.x >> 5] = t1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < kSp2Threads / 32; ++w) {
            s0 += part[0][w];
            s1 += part[1][w];
        }
        square = fabs(s1 - ne) < fabs(2.0 * s0 - s1 - ne);
    }
    __syncthreads();
    const bool sq = square != 0;
    const size_t nn = (size_t)n * n;
    for (size_t k = (size_t)blockIdx.x * kSp2Threads + threadIdx.x; k < nn; k += (size_t)gridDim.x * kSp2Threads)
        Yout[k] = sq ? Y2[k] : 2.0 * Y[k] - Y2[k];
}

// The GEMM of the SP2 steps is cuBLAS's DGEMM, one handle per device, shared by every
// stream (the enqueue is serialised by a mutex).  The handle runs without a workspace,
// so that calls on different streams share no scratch memory and a call inside a
// stream capture allocates nothing; it is created by the first call on the device,
// which must come before any capture.
struct BlasHandles {
    std::mutex mu;
    std::map<int, cublasHandle_t> by_device;
};

static BlasHandles& blas_handles() {
    static BlasHandles b;
    return b;
}

// The current device's handle, bound to `s` with no workspace.  Caller holds the mutex.
static int blas_on(cudaStream_t s, cublasHandle_t* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return QK_ERR_CUDA;
    auto& m = blas_handles().by_device;
    auto it = m.find(dev);
    if (it == m.end()) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (s && cudaStreamIsCapturing(s, &cap) != cudaSuccess) return QK_ERR_CUDA;
        if (cap != cudaStreamCaptureStatusNone) return QK_ERR_NOT_READY;   // creating it would allocate
        cublasHandle_t h = nullptr;
        if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return QK_ERR_CUDA;
        it = m.emplace(dev, h).first;
    }
    if (cublasSetStream(it->second, s) != CUBLAS_STATUS_SUCCESS ||
        cublasSetWorkspace(it->second, nullptr, 0) != CUBLAS_STATUS_SUCCESS)
        return QK_ERR_CUDA;
    *out = it->second;
    return QK_OK;
}

}  // namespace qk

extern "C" int qk_sp2_run(double* Ya, double* Yb, double* Y2, int n, double nocc, int steps, void* stream) {
    if (!Ya || !Yb || !Y2 || n < 1 || steps < 0 || Ya == Yb || Ya == Y2 || Yb == Y2) return QK_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nn = (size_t)n * n;
    const int grid = (int)std::min<size_t>(4 * 148, (nn + qk::kSp2Threads - 1) / qk::kSp2Threads);
    std::lock_guard<std::mutex> guard(qk::blas_handles().mu);
    cublasHandle_t h = nullptr;
    const int st = qk::blas_on(s, &h);
    if (st != QK_OK) return st;
    const double one = 1.0, zero = 0.0;
    double* cur = Ya;
    double* nxt = Yb;
    for (int k = 0; k < steps; ++k) {
        // row-major Y2 = Y Y is column-major Y2^T = Y^T Y^T: the same call
        if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, cur, n, cur, n, &zero, Y2, n) !=
            CUBLAS_STATUS_SUCCESS)
            return QK_ERR_CUDA;
        qk::sp2_step_kernel<<<grid, qk::kSp2Threads, 0, s>>>(cur, Y2, nxt, n, nocc);
        if (cudaGetLastError() != cudaSuccess) return QK_ERR_CUDA;
        std::swap(cur, nxt);
    }
    return QK_OK;
}

extern "C" int qk_sp2_step(const double* Y, const double* Y2, double* Yout, int n, double nocc, void* stream) {
    if (!Y || !Y2 || !Yout || n < 1 || Yout == Y || Yout == Y2) return QK_ERR_INVALID_ARG;
    const size_t nn = (size_t)n * n;
    const int grid = (int)std::min<size_t>(4 * 148, (nn + qk::kSp2Threads - 1) / qk::kSp2Threads);
    qk::sp2_step_kernel<<<grid, qk::kSp2Threads, 0, (cudaStream_t)stream>>>(Y, Y2, Yout, n, nocc);
    return cudaGetLastError() == cudaSuccess ? QK_OK : QK_ERR_CUDA;
}

extern "C" int qk_small_solve(const double* A, const double* b, int n, double* x, int* ok, void* stream) {
    if (!A || !b || !x || !ok || n < 1 || n > qk::kSmallSolveMax) return QK_ERR_INVALID_ARG;
    qk::small_solve_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(A, b, n, x, ok);
    return cudaGetLastError() == cudaSuccess ? QK_OK : QK_ERR_CUDA;
}
