// get_modes on the device.
//
// Reference: get_modes(dynmat, num_rigid_translation = 3)   src/dynmat.jl:123-141
//     eig = eigen(Hermitian(dynmat))          ascending eigenvalues, orthonormal vectors
//     idx = sortperm(abs.(eig.values))        stable sort of |λ|
//     eig.values[idx[1:num_rigid_translation]] .= 0.0
//
// Here the symmetric FP64 eigenproblem is solved by cuSOLVER's divide-and-
// conquer `syevd` on the caller's stream (upper triangle, as Hermitian(A)
// defaults to), the rigid-translation eigenvalues are zeroed by a small kernel
// that computes each eigenvalue's position in the stable order of |λ|, and the
// eigenvectors are optionally also written as FP32 — the φ operand of mcc3 —
// so a snapshot's modes never leave the device.
//
// cuSOLVER is opened with dlopen on first use: a process that already holds a
// libcusolver (a framework that loaded its own copy) shares it, and the rest of
// the library does not depend on it being installed.
#include <dlfcn.h>
#include <cusolverDn.h>

#include <mutex>
#include <string>

#include "fcb200_internal.cuh"

namespace fcb {
namespace {

struct SolverLib {
    bool tried = false;
    void* so = nullptr;
    decltype(&cusolverDnCreate) create = nullptr;
    decltype(&cusolverDnDestroy) destroy = nullptr;
    decltype(&cusolverDnSetStream) set_stream = nullptr;
    decltype(&cusolverDnDsyevd_bufferSize) buffer_size = nullptr;
    decltype(&cusolverDnDsyevd) syevd = nullptr;
};

SolverLib g_solver;
std::mutex g_solver_mu;

int load_solver() {
    std::lock_guard<std::mutex> lock(g_solver_mu);
    if (!g_solver.tried) {
        g_solver.tried = true;
        const char* names[] = {"libcusolver.so.11", "libcusolver.so"};
        for (const char* nm : names) {
            g_solver.so = dlopen(nm, RTLD_NOW | RTLD_LOCAL);
            if (g_solver.so) break;
        }
        if (g_solver.so) {
            g_solver.create = reinterpret_cast<decltype(g_solver.create)>(dlsym(g_solver.so, "cusolverDnCreate"));
            g_solver.destroy = reinterpret_cast<decltype(g_solver.destroy)>(dlsym(g_solver.so, "cusolverDnDestroy"));
            g_solver.set_stream =
                reinterpret_cast<decltype(g_solver.set_stream)>(dlsym(g_solver.so, "cusolverDnSetStream"));
            g_solver.buffer_size = reinterpret_cast<decltype(g_solver.buffer_size)>(
                dlsym(g_solver.so, "cusolverDnDsyevd_bufferSize"));
            g_solver.syevd = reinterpret_cast<decltype(g_solver.syevd)>(dlsym(g_solver.so, "cusolverDnDsyevd"));
        }
    }
    if (!g_solver.so || !g_solver.create || !g_solver.destroy || !g_solver.set_stream || !g_solver.buffer_size ||
        !g_solver.syevd)
        return set_error(FCB_ERR_UNSUPPORTED, "get_modes: libcusolver could not be opened");
    return FCB_OK;
}

// Position of eigenvalue i in sortperm(abs.(w)) (stable; NaN sorts last, as
// Julia's isless does) is below k  ⇒  w[i] = 0.  One block; `n` bytes of flags
// in shared memory so that every rank is computed from the unmodified values.
__global__ void zero_rigid_kernel(double* __restrict__ w, int n, int k) {
    extern __shared__ unsigned char zero_flag[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double ai = fabs(w[i]);
        const bool nan_i = isnan(ai);
        int rank = 0;
        for (int j = 0; j < n && rank < k; ++j) {
            const double aj = fabs(w[j]);
            const bool nan_j = isnan(aj);
            bool before;
            if (nan_i)
                before = !nan_j || j < i;
            else
                before = !nan_j && (aj < ai || (aj == ai && j < i));
            rank += before ? 1 : 0;
        }
        zero_flag[i] = rank < k ? 1 : 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (zero_flag[i]) w[i] = 0.0;
}

__global__ void to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride) b[t] = (float)a[t];
}

int solver_error(const char* what, int code) {
    return set_error(FCB_ERR_CUDA, std::string("get_modes: ") + what + " returned cusolver status " +
                                       std::to_string(code));
}

}  // namespace

void modes_release(fcb200_context* h) {
    if (h->solver && g_solver.destroy) g_solver.destroy(static_cast<cusolverDnHandle_t>(h->solver));
    h->solver = nullptr;
}

}  // namespace fcb

using namespace fcb;

extern "C" {

int fcb200_get_modes(fcb200_handle h, const double* dynmat, int64_t n, int num_rigid, double* freqs_sq,
                     double* modes, float* phi32, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (!dynmat || !freqs_sq) return set_error(FCB_ERR_ARG, "dynmat and freqs_sq must not be NULL");
    if (n < 1 || n > 3 * 4096) return set_error(FCB_ERR_ARG, "get_modes: n must be in [1, 12288]");
    if (num_rigid < 0 || num_rigid > n) return set_error(FCB_ERR_ARG, "num_rigid_translation must be in [0, n]");
    FCB_TRY(load_solver());
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!h->solver) {
        cusolverDnHandle_t sh = nullptr;
        const cusolverStatus_t st = g_solver.create(&sh);
        if (st != CUSOLVER_STATUS_SUCCESS) return solver_error("cusolverDnCreate", (int)st);
        h->solver = sh;
    }
    cusolverDnHandle_t sh = static_cast<cusolverDnHandle_t>(h->solver);
    {
        const cusolverStatus_t st = g_solver.set_stream(sh, s);
        if (st != CUSOLVER_STATUS_SUCCESS) return solver_error("cusolverDnSetStream", (int)st);
    }
    const size_t nn = (size_t)n * (size_t)n;
    // A: overwritten by the eigenvectors (the caller's `modes` when it is device memory).
    double* a = nullptr;
    const bool modes_dev = modes && is_device_ptr(modes);
    if (modes_dev) {
        a = modes;
    } else {
        FCB_TRY(h->eig_a.ensure(sizeof(double) * nn));
        a = h->eig_a.as<double>();
    }
    if (a != dynmat)
        FCB_CUDA(cudaMemcpyAsync(a, dynmat, sizeof(double) * nn, cudaMemcpyDefault, s));
    const bool w_dev = is_device_ptr(freqs_sq);
    double* w = nullptr;
    if (w_dev) {
        w = freqs_sq;
    } else {
        FCB_TRY(h->eig_w.ensure(sizeof(double) * (size_t)n));
        w = h->eig_w.as<double>();
    }
    int lwork = 0;
    {
        const cusolverStatus_t st = g_solver.buffer_size(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER,
                                                         (int)n, a, (int)n, w, &lwork);
        if (st != CUSOLVER_STATUS_SUCCESS) return solver_error("cusolverDnDsyevd_bufferSize", (int)st);
    }
    FCB_TRY(h->eig_work.ensure(sizeof(double) * (size_t)(lwork > 0 ? lwork : 1) + 256));
    double* work = h->eig_work.as<double>();
    int* info = reinterpret_cast<int*>(reinterpret_cast<char*>(work) + sizeof(double) * (size_t)(lwork > 0 ? lwork : 1));
    {
        const cusolverStatus_t st =
            g_solver.syevd(sh, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, (int)n, a, (int)n, w, work, lwork, info);
        if (st != CUSOLVER_STATUS_SUCCESS) return solver_error("cusolverDnDsyevd", (int)st);
    }
    if (num_rigid > 0) {
        zero_rigid_kernel<<<1, 1024, (size_t)n, s>>>(w, (int)n, num_rigid);
        FCB_CUDA(cudaGetLastError());
    }
    if (phi32) {
        float* f = phi32;
        const bool f_dev = is_device_ptr(phi32);
        if (!f_dev) {
            FCB_TRY(h->phi_f32.ensure(sizeof(float) * nn));
            f = h->phi_f32.as<float>();
        }
        const int64_t blocks = (int64_t)(nn + 255) / 256;
        to_f32_kernel<<<(unsigned)(blocks < 8 * h->sm_count ? blocks : 8 * h->sm_count), 256, 0, s>>>(a, f, (int64_t)nn);
        FCB_CUDA(cudaGetLastError());
        if (!f_dev) FCB_CUDA(cudaMemcpyAsync(phi32, f, sizeof(float) * nn, cudaMemcpyDeviceToHost, s));
    }
    if (modes && !modes_dev) FCB_CUDA(cudaMemcpyAsync(modes, a, sizeof(double) * nn, cudaMemcpyDeviceToHost, s));
    if (!w_dev) FCB_CUDA(cudaMemcpyAsync(freqs_sq, w, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s));
    // The convergence flag decides whether the outputs mean anything: read it.
    int info_h = 0;
    FCB_CUDA(cudaMemcpyAsync(&info_h, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    FCB_CUDA(cudaStreamSynchronize(s));
    if (info_h != 0)
        return set_error(FCB_ERR_CUDA, "get_modes: syevd did not converge (info = " + std::to_string(info_h) + ")");
    return FCB_OK;
}

}  // extern "C"
