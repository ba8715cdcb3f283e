// fcb200_third_order_lj_noalloc: LJ IFC3 assembly that allocates no device
// memory at all.
//
// Why it exists: some callers cannot let a library call cudaMalloc/cudaFree.
// A Julia host (the ccall shim) keeps every device buffer in CUDA.jl's own
// memory pool, and allocations made behind its back are invisible to that
// pool's accounting and to its out-of-memory handling; applications that size
// all device memory once at start-up have the same constraint.  cudaFree also
// synchronises the whole device, which stalls a caller that keeps several
// streams busy.  This entry point therefore takes only caller buffers and keeps
// its scratch (pair tables, within-cutoff flags, ASR self blocks and the box)
// in one fixed device array defined in this file.
//
// Limits and behaviour:
//  * at most FCB_NOALLOC_MAX_ATOMS atoms; larger systems are rejected with
//    FCB_ERR_ARG before any device work;
//  * every GPU that loads the library holds the array (about 14.3 MB) until the
//    process exits;
//  * all calls share the array and it keeps the previous call's contents.
//    Nothing in it has to start at zero: every entry a call reads is written
//    earlier in the same call (all N*N flags, then only flagged pair blocks,
//    then all self blocks).  Calls whose work overlaps on the GPU (different
//    streams, or different host threads) race on the array and must be
//    serialised by the caller;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current, and so does the first
//    call after that device's context was torn down and created again (for
//    example by cudaDeviceReset): the address is cached per CUDA context.
//    Make that first call before any stream capture begins.
#include <cuda.h>

#include <mutex>

#include "fcb200_internal.cuh"

namespace fcb {
namespace {

constexpr int64_t kMaxAtoms = FCB_NOALLOC_MAX_ATOMS;
constexpr size_t kBoxOff = 0;                                                      // 3 doubles
constexpr size_t kTOff = 256;                                                      // N² × 27 doubles
constexpr size_t kSOff = kTOff + sizeof(double) * 27 * kMaxAtoms * kMaxAtoms;    // N × 27 doubles
constexpr size_t kFlagOff = kSOff + sizeof(double) * 27 * kMaxAtoms;              // N² bytes
constexpr size_t kScratchBytes = ((kFlagOff + kMaxAtoms * kMaxAtoms + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct ScratchSlot {
    CUcontext ctx = nullptr;  // context the address belongs to
    void* addr = nullptr;
};
ScratchSlot g_slot[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// The driver's cuCtxGetCurrent, through the runtime (no link-time libcuda).
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
        tried = true;
    }
    return fn;
}

// Device address of the scratch array in the current device's context, looked
// up on the first call in that context (a context created anew after a reset
// gets a fresh lookup).  While no context is current on the calling thread yet,
// or without the driver entry point, it is looked up on every call;
// cudaGetSymbolAddress itself makes the device's primary context current.
int scratch_address(void** out) {
    int dev = 0;
    FCB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(FCB_ERR_ARG, "device index out of range");
    CUcontext ctx = nullptr;
    CtxGetCurrentFn get = ctx_get_current();
    const bool known = get != nullptr && get(&ctx) == CUDA_SUCCESS && ctx != nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    ScratchSlot& slot = g_slot[dev];
    if (!known || slot.addr == nullptr || slot.ctx != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
        slot.addr = p;
        slot.ctx = known ? ctx : nullptr;
    }
    *out = slot.addr;
    return FCB_OK;
}

// The three box lengths, passed by value, written into the scratch array.
__global__ void put_box_kernel(double* d_box, double bx, double by, double bz) {
    if (threadIdx.x == 0) {
        d_box[0] = bx;
        d_box[1] = by;
        d_box[2] = bz;
    }
}

int require_device(const void* p, const char* name) {
    if (p != nullptr && !is_device_ptr(p))
        return set_error(FCB_ERR_ARG, std::string(name) +
                                          " must be device memory (this entry point stages nothing on the device)");
    return FCB_OK;
}

}  // namespace
}  // namespace fcb

using namespace fcb;

extern "C" int fcb200_third_order_lj_noalloc(const double* pos, int64_t n_atoms, const double* box, double sigma,
                                             double eps, double r_cut, double tol, const double* masses,
                                             double* psi_out, float* psi32_mw_out, int flags, void* stream) {
    const bool weighted = (flags & FCB_PSI_MASS_WEIGHTED) != 0;
    if (pos == nullptr || box == nullptr) return set_error(FCB_ERR_ARG, "pos and box must not be NULL");
    if (n_atoms < 1) return set_error(FCB_ERR_ARG, "n_atoms must be >= 1");
    if (n_atoms > kMaxAtoms)
        return set_error(FCB_ERR_ARG, "n_atoms = " + std::to_string(n_atoms) +
                                          " exceeds the fixed scratch of fcb200_third_order_lj_noalloc (max " +
                                          std::to_string(kMaxAtoms) + " atoms); use fcb200_third_order_lj");
    if ((weighted || psi32_mw_out != nullptr) && masses == nullptr)
        return set_error(FCB_ERR_ARG, "masses are required for mass weighting");
    if (psi_out == nullptr && psi32_mw_out == nullptr) return set_error(FCB_ERR_ARG, "no output buffer given");
    if (!(r_cut > 0.0)) return set_error(FCB_ERR_ARG, "r_cut must be positive");
    if (is_device_ptr(box)) return set_error(FCB_ERR_ARG, "box must be a host array of 3 doubles");
    for (int d = 0; d < 3; ++d) {
        if (!(box[d] > 0.0)) return set_error(FCB_ERR_ARG, "box lengths must be positive");
        if (!(r_cut < box[d])) return set_error(FCB_ERR_CUTOFF, "Cutoff larger than L/2 (r_cut must be < box length)");
    }
    FCB_TRY(require_device(pos, "pos"));
    FCB_TRY(require_device(masses, "masses"));
    FCB_TRY(require_device(psi_out, "psi_out"));
    FCB_TRY(require_device(psi32_mw_out, "psi32_mw_out"));

    void* base = nullptr;
    FCB_TRY(scratch_address(&base));
    int dev = 0, sms = 0;
    FCB_CUDA(cudaGetDevice(&dev));
    FCB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(base);
    double* d_box = reinterpret_cast<double*>(b + kBoxOff);
    double* T = reinterpret_cast<double*>(b + kTOff);
    double* S = reinterpret_cast<double*>(b + kSOff);
    uint8_t* flag = reinterpret_cast<uint8_t*>(b + kFlagOff);
    put_box_kernel<<<1, 32, 0, s>>>(d_box, box[0], box[1], box[2]);
    FCB_CUDA(cudaGetLastError());
    FCB_TRY(lj_pair_tables_raw(T, flag, S, pos, n_atoms, d_box, sigma, eps, r_cut, s));
    AssemblyOut out;
    out.psi64 = psi_out;
    out.psi64_weighted = weighted;
    out.psi32 = psi32_mw_out;
    FCB_TRY(ifc3_dense_write_raw(T, flag, S, sms, n_atoms, tol, masses, out, s));
    return FCB_OK;
}
