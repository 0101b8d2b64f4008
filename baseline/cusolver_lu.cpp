// Library baseline for the FP64 solve: cuSOLVER LU with partial pivoting and
// the multi-right-hand-side solve, called the way the reference's
// lu_solve_full calls it (solver.cu:87-142): the row-major Z is handed over
// as the column-major Z^T, factored in place, and Z X = B is solved with
// the transposed operation.  The 64-bit API (cusolverDnXgetrf / Xgetrs) is
// used because n^2 exceeds 2^31 at 2N = 61440; the reference calls the
// 32-bit cusolverDnZgetrf.  Benchmark infrastructure: nothing in the
// library links it.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdint>
#include <cstdlib>

extern "C" {

// Z: device, n x n complex128 row-major (overwritten with the factors of Z^T).
// B: device, nrhs columns of length n at stride ldb (overwritten with X).
// Returns 0, or -1 (CUDA error), -2 (cuSOLVER error), or info > 0 (a zero
// pivot) / info < 0 (bad argument) as cuSOLVER reports it.
int cs_lu_solve(void* stream, void* Z, int64_t n, void* B, int64_t ldb, int64_t nrhs) {
    cusolverDnHandle_t h = nullptr;
    cusolverDnParams_t p = nullptr;
    int64_t* ipiv = nullptr;
    int* dinfo = nullptr;
    void* dwork = nullptr;
    void* hwork = nullptr;
    int rc = 0, info = 0;
    size_t dbytes = 0, hbytes = 0;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return -2;
    if (cusolverDnSetStream(h, (cudaStream_t)stream) != CUSOLVER_STATUS_SUCCESS ||
        cusolverDnCreateParams(&p) != CUSOLVER_STATUS_SUCCESS) { rc = -2; goto done; }
    if (cudaMalloc(&ipiv, sizeof(int64_t) * n) != cudaSuccess ||
        cudaMalloc(&dinfo, sizeof(int)) != cudaSuccess) { rc = -1; goto done; }
    if (cusolverDnXgetrf_bufferSize(h, p, n, n, CUDA_C_64F, Z, n, CUDA_C_64F, &dbytes, &hbytes) !=
        CUSOLVER_STATUS_SUCCESS) { rc = -2; goto done; }
    if (dbytes && cudaMalloc(&dwork, dbytes) != cudaSuccess) { rc = -1; goto done; }
    if (hbytes && !(hwork = std::malloc(hbytes))) { rc = -1; goto done; }
    if (cusolverDnXgetrf(h, p, n, n, CUDA_C_64F, Z, n, ipiv, CUDA_C_64F, dwork, dbytes, hwork, hbytes,
                         dinfo) != CUSOLVER_STATUS_SUCCESS) { rc = -2; goto done; }
    if (cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) { rc = -1; goto done; }
    if (info != 0) { rc = info; goto done; }
    if (cusolverDnXgetrs(h, p, CUBLAS_OP_T, n, nrhs, CUDA_C_64F, Z, n, ipiv, CUDA_C_64F, B, ldb, dinfo) !=
        CUSOLVER_STATUS_SUCCESS) { rc = -2; goto done; }
    if (cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) { rc = -1; goto done; }
    rc = info;
done:
    if (dwork) cudaFree(dwork);
    if (hwork) std::free(hwork);
    if (ipiv) cudaFree(ipiv);
    if (dinfo) cudaFree(dinfo);
    if (p) cusolverDnDestroyParams(p);
    if (h) cusolverDnDestroy(h);
    return rc;
}

}  // extern "C"
