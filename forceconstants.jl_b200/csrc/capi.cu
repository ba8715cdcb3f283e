// extern "C" entry points of libfcb200 (declared in include/fcb200.h).
//
// The host side here only validates arguments, stages host buffers, sizes the
// handle's scratch and sequences kernel launches on the caller's stream; all
// arithmetic runs in the kernels of lj_assembly.cu, mode_product_*.cu and
// mcc3.cu.
#include <cstdio>
#include <cstring>
#include <string>

#include <vector>

#include "fcb200_internal.cuh"

namespace fcb {

namespace {
thread_local std::string t_msg = "no error";
thread_local int t_code = FCB_OK;
}  // namespace

int set_error(int code, const std::string& msg) {
    t_code = code;
    t_msg = msg;
    return code;
}

int cuda_error(cudaError_t e, const char* what) {
    return set_error(e == cudaErrorMemoryAllocation ? FCB_ERR_OOM : FCB_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

int Buf::ensure(size_t need) {
    if (need <= bytes && p != nullptr) return FCB_OK;
    release();
    if (need == 0) return FCB_OK;
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        cudaGetLastError();
        return set_error(FCB_ERR_OOM, "device allocation of " + std::to_string(need) + " bytes refused: " +
                                          cudaGetErrorString(e));
    }
    bytes = need;
    return FCB_OK;
}

void Buf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

bool is_device_ptr(const void* ptr) {
    if (ptr == nullptr) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

namespace {

// Device view of a caller buffer: the pointer itself when it is device memory,
// otherwise a handle scratch buffer (filled from the host when `upload`).
template <class T>
int device_view(Buf& scratch, const T* user, size_t count, bool upload, cudaStream_t s, T** out) {
    if (user == nullptr) {
        *out = nullptr;
        return FCB_OK;
    }
    if (is_device_ptr(user)) {
        *out = const_cast<T*>(user);
        return FCB_OK;
    }
    FCB_TRY(scratch.ensure(sizeof(T) * count));
    if (upload) FCB_CUDA(cudaMemcpyAsync(scratch.p, user, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    *out = scratch.as<T>();
    return FCB_OK;
}

int check_status(fcb200_context* h, cudaStream_t s) {
    FCB_CUDA(cudaStreamSynchronize(s));
    int st = 0;
    FCB_CUDA(cudaMemcpy(&st, h->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != DEV_OK) {
        int zero = 0;
        cudaMemcpy(h->d_status, &zero, sizeof(int), cudaMemcpyHostToDevice);
        if (st == DEV_SPARSE_OVERFLOW)
            return set_error(FCB_ERR_ARG, "a neighbourhood grew past the capacity fixed in advance (a batch's: set "
                                          "the snapshot's positions again so that the batch is re-planned; or "
                                          "fcb200_set_neighbour_capacity's); K3 is invalid");
        if (st == DEV_FD_OVERFLOW)
            return set_error(FCB_ERR_UNSUPPORTED, "finite differences: more than 128 atoms within the SW cutoff of "
                                                  "the displaced atoms");
        return set_error(FCB_ERR_TIMEOUT, "a bounded device-side wait gave up (code " + std::to_string(st) +
                                              "); the kernel returned early and its output is invalid");
    }
    return FCB_OK;
}

int esz_of(int kind) { return kind == 1 ? 2 : 4; }

int validate_lj(const double* pos, int64_t N, const double* box, double r_cut, const double* masses,
                bool need_masses) {
    if (pos == nullptr || box == nullptr) return set_error(FCB_ERR_ARG, "pos and box must not be NULL");
    if (N < 1) return set_error(FCB_ERR_ARG, "n_atoms must be >= 1");
    if (N > 4096) return set_error(FCB_ERR_ARG, "n_atoms > 4096 (dense n³ tensor would exceed device memory)");
    if (need_masses && masses == nullptr) return set_error(FCB_ERR_ARG, "masses are required for mass weighting");
    if (!(r_cut > 0.0)) return set_error(FCB_ERR_ARG, "r_cut must be positive");
    return FCB_OK;
}

int check_cutoff(const double* box_host) {
    for (int d = 0; d < 3; ++d)
        if (!(box_host[d] > 0.0)) return set_error(FCB_ERR_ARG, "box lengths must be positive");
    return FCB_OK;
}

// Reads the 3 box lengths to the host (the r_cut < L check of
// third_order_analytical.jl:7 is a host-side status, not a device assert).
int box_to_host(const double* box, double out[3]) {
    if (is_device_ptr(box)) {
        FCB_CUDA(cudaMemcpy(out, box, 3 * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
        memcpy(out, box, 3 * sizeof(double));
    }
    return FCB_OK;
}

struct Mcc3Operand {
    const float* f32 = nullptr;  // FP32 Ψ with lda = n
    const void* hi = nullptr;    // split planes with lda = n_pad
    const void* lo = nullptr;
};

// P1..P3 on device buffers.  `emit` receives each finished slab of the last
// mode axis when slab > 0 (used by the blocked / host-output forms).
// Symmetric tiles (ModeProduct::sym) are used when the row layout keeps 8
// consecutive rows contiguous and aligned (the vector epilogue).
static bool sym_ok(const ModeProduct& mp) { return mp.F % 8 == 0 && mp.F_pad % 8 == 0 && mp.ldd % 8 == 0; }

// `sym`: Ψ is symmetric in all three indices (an assembled IFC3) and the three
// mode windows coincide, so U2 is symmetric in its two mode indices and K3 in
// its last two; the tensor-core P2 and P3 then compute only one triangle of
// tiles and mirror the rest.
int run_mcc3(fcb200_context* h, int precision, const Mcc3Operand& psi, const float* d_phi, int64_t n,
             int64_t n_lo, int64_t n_hi, int64_t m_lo, int64_t m_hi, int64_t l_lo, int64_t l_hi, float* d_k3,
             cudaStream_t s, bool sym = false) {
    const int64_t Mn = n_hi - n_lo, Mm = m_hi - m_lo, Ml = l_hi - l_lo;
    if (precision == FCB_MCC3_FP32) {
        FCB_TRY(h->u1_f32.ensure(sizeof(float) * n * n * Mn));
        FCB_TRY(h->u2_f32.ensure(sizeof(float) * n * Mn * Mm));
        phase_mark(h, s, 3);
        ModeProduct p1{n * n, n, Mn, n, n, n, n, n * n};
        FCB_TRY(mode_product_f32(psi.f32, d_phi + n * n_lo, h->u1_f32.as<float>(), p1, s));
        phase_mark(h, s, 4);
        ModeProduct p2{n * Mn, n, Mm, n, n, n, n, n * Mn};
        FCB_TRY(mode_product_f32(h->u1_f32.as<float>(), d_phi + n * m_lo, h->u2_f32.as<float>(), p2, s));
        phase_mark(h, s, 5);
        ModeProduct p3{Mn * Mm, n, Ml, n, n, Mn * Mm, Mn * Mm, Mn * Mm};
        FCB_TRY(mode_product_f32(h->u2_f32.as<float>(), d_phi + n * l_lo, d_k3, p3, s));
        phase_mark(h, s, 6);
        return FCB_OK;
    }
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    const int64_t np = pad_for(kind, n);
    const size_t esz = esz_of(kind);
    // φ planes for all n columns: [mode][n_pad]
    FCB_TRY(h->phi_hi.ensure(esz * np * n));
    FCB_TRY(h->phi_lo.ensure(esz * np * n));
    FCB_TRY(split_operand(d_phi, n, n, n, h->phi_hi.p, h->phi_lo.p, np, kind, s));
    phase_mark(h, s, 3);
    FCB_TRY(h->u1_hi.ensure(esz * np * n * Mn));
    FCB_TRY(h->u1_lo.ensure(esz * np * n * Mn));
    FCB_TRY(h->u2_hi.ensure(esz * np * Mn * Mm));
    FCB_TRY(h->u2_lo.ensure(esz * np * Mn * Mm));
    auto plane = [&](const Buf& b, int64_t mode) {
        return static_cast<const void*>(static_cast<const uint8_t*>(b.p) + esz * np * mode);
    };
    ModeProduct p1{n * n, n, Mn, np, np, n, np, np * n};
    FCB_TRY(mode_product_tc(h, kind, psi.hi, psi.lo, plane(h->phi_hi, n_lo), plane(h->phi_lo, n_lo), h->u1_hi.p,
                            h->u1_lo.p, kind, p1, s));
    phase_mark(h, s, 4);
    sym = sym && n_lo == m_lo && m_lo == l_lo && Mn == Mm && Mm == Ml;
    ModeProduct p2{n * Mn, n, Mm, np, np, n, np, np * Mn};
    p2.sym = sym && sym_ok(p2);
    FCB_TRY(mode_product_tc(h, kind, h->u1_hi.p, h->u1_lo.p, plane(h->phi_hi, m_lo), plane(h->phi_lo, m_lo),
                            h->u2_hi.p, h->u2_lo.p, kind, p2, s));
    phase_mark(h, s, 5);
    ModeProduct p3{Mn * Mm, n, Ml, np, np, Mn * Mm, Mn * Mm, Mn * Mm};
    ModeProduct p3s{Mn * Mm, n, Ml, np, np, Mn, Mn, Mn * Mm};  // rows p + Mn·q: K3[p,q,s] = K3[p,s,q]
    p3s.sym = true;
    if (sym && sym_ok(p3s)) p3 = p3s;
    FCB_TRY(mode_product_tc(h, kind, h->u2_hi.p, h->u2_lo.p, plane(h->phi_hi, l_lo), plane(h->phi_lo, l_lo), d_k3,
                            nullptr, 0, p3, s));
    phase_mark(h, s, 6);
    return FCB_OK;
}

int check_precision(int precision) {
    if (precision != FCB_MCC3_FP32 && precision != FCB_MCC3_BF16X3 && precision != FCB_MCC3_TF32X3)
        return set_error(FCB_ERR_ARG, "unknown mcc3 precision mode");
    return FCB_OK;
}

// Stage the mass-weighted Ψ operand for a given precision from an FP32 Ψ.
int psi_operand_from_f32(fcb200_context* h, int precision, const float* d_psi, int64_t n, cudaStream_t s,
                         Mcc3Operand* op) {
    if (precision == FCB_MCC3_FP32) {
        op->f32 = d_psi;
        return FCB_OK;
    }
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    const int64_t np = pad_for(kind, n);
    FCB_TRY(h->psi_hi.ensure((size_t)esz_of(kind) * np * n * n));
    FCB_TRY(h->psi_lo.ensure((size_t)esz_of(kind) * np * n * n));
    FCB_TRY(split_operand(d_psi, n * n, n, n, h->psi_hi.p, h->psi_lo.p, np, kind, s));
    op->hi = h->psi_hi.p;
    op->lo = h->psi_lo.p;
    return FCB_OK;
}

}  // namespace
}  // namespace fcb

using namespace fcb;

extern "C" {

int fcb200_version(void) { return 100; }

int fcb200_last_error(char* buf, size_t len) {
    if (buf && len) {
        strncpy(buf, t_msg.c_str(), len - 1);
        buf[len - 1] = '\0';
    }
    return t_code;
}

int fcb200_create(fcb200_handle* out, int device) {
    if (!out) return set_error(FCB_ERR_ARG, "out must not be NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_error(FCB_ERR_UNSUPPORTED, "no CUDA device available");
    }
    if (device < 0 || device >= count) return set_error(FCB_ERR_ARG, "device index out of range");
    FCB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FCB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_error(FCB_ERR_UNSUPPORTED, std::string("fcb200 requires an sm_100 (B200) device, found ") + prop.name);
    auto* h = new fcb200_context();
    h->device = device;
    h->sm_count = prop.multiProcessorCount;
    if (cudaMalloc(&h->d_status, sizeof(int)) != cudaSuccess) {
        delete h;
        return set_error(FCB_ERR_OOM, "status word allocation failed");
    }
    cudaMemset(h->d_status, 0, sizeof(int));
    cudaStreamCreateWithFlags(&h->aux_stream, cudaStreamNonBlocking);
    for (auto& ev : h->ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    *out = h;
    return FCB_OK;
}

int fcb200_trim(fcb200_handle h) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    cudaSetDevice(h->device);
    Buf* bufs[] = {&h->pos, &h->box, &h->masses, &h->pair_t, &h->pair_flag, &h->self_t, &h->psi_stage,
                   &h->phi_f32, &h->phi_hi, &h->phi_lo, &h->psi_hi, &h->psi_lo, &h->u1_hi, &h->u1_lo,
                   &h->u2_hi, &h->u2_lo, &h->u1_f32, &h->u2_f32, &h->psi_f32, &h->k3_stage[0],
                   &h->k3_stage[1], &h->k3_full, &h->ifc2, &h->sw_ints, &h->sw_nbr_r, &h->sw_pair_off, &h->sw_blk3,
                   &h->sw_blk2, &h->sw_atoms, &h->sw_place, &h->sw_col_off, &h->sw_col_items, &h->sw_cursor,
                   &h->sw_asr_off, &h->sw_asr_items, &h->sw_asr, &h->adj_phiT, &h->adj_w_hi, &h->adj_w_lo,
                   &h->adj_pairs, &h->adj_G, &h->adj_scal, &h->adj_w32, &h->adj_dpos, &h->adj_w64,
                   &h->adj_phiT64, &h->eig_a, &h->eig_w,
                   &h->eig_work, &h->sp_ints, &h->sp_coef, &h->phik_hi, &h->phik_lo, &h->fd_elems, &h->fd_out};
    for (Buf* b : bufs) b->release();
    return FCB_OK;
}

int fcb200_destroy(fcb200_handle h) {
    if (!h) return FCB_OK;
    cudaSetDevice(h->device);
    fcb200_trim(h);
    modes_release(h);
    if (h->owns_tune) delete h->tune;
    if (h->d_status) cudaFree(h->d_status);
    if (h->h_pinned) cudaFreeHost(h->h_pinned);
    if (h->aux_stream) cudaStreamDestroy(h->aux_stream);
    for (auto& e : h->pev)
        if (e) cudaEventDestroy(e);
    for (auto& ev : h->ev)
        if (ev) cudaEventDestroy(ev);
    delete h;
    return FCB_OK;
}

int fcb200_synchronize(fcb200_handle h, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    return check_status(h, static_cast<cudaStream_t>(stream));
}

int fcb200_set_wait_limit(fcb200_handle h, int64_t limit_ns) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    h->wait_limit_ns = limit_ns > 0 ? (uint64_t)limit_ns : 2000000000ull;
    return FCB_OK;
}

int fcb200_set_neighbour_capacity(fcb200_handle h, int cap) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (cap < 0) return set_error(FCB_ERR_ARG, "the neighbour capacity must be >= 0");
    h->fixed_cap = cap;
    return FCB_OK;
}

int fcb200_set_profiling(fcb200_handle h, int enable) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    cudaSetDevice(h->device);
    if (enable && !h->pev[0])
        for (auto& e : h->pev) FCB_CUDA(cudaEventCreate(&e));
    h->profiling = enable != 0;
    return FCB_OK;
}

int fcb200_phase_times(fcb200_handle h, double* ms, int max_phases) {
    if (!h || !ms) return set_error(FCB_ERR_ARG, "NULL argument");
    cudaSetDevice(h->device);
    int k = 0;
    for (int i = 0; i + 1 < fcb200_context::kMarks && k < max_phases; ++i, ++k) {
        ms[k] = -1.0;
        if (h->profiling && h->marked[i] && h->marked[i + 1]) {
            float t = 0.f;
            FCB_CUDA(cudaEventSynchronize(h->pev[i + 1]));
            FCB_CUDA(cudaEventElapsedTime(&t, h->pev[i], h->pev[i + 1]));
            ms[k] = t;
        }
    }
    return FCB_OK;
}

int fcb200_third_order_lj(fcb200_handle h, const double* pos, int64_t N, const double* box, double sigma,
                          double eps, double r_cut, double tol, const double* masses, double* psi_out,
                          float* psi32_mw_out, int flags, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    const bool weighted = (flags & FCB_PSI_MASS_WEIGHTED) != 0;
    FCB_TRY(validate_lj(pos, N, box, r_cut, masses, weighted || psi32_mw_out != nullptr));
    if (!psi_out && !psi32_mw_out) return set_error(FCB_ERR_ARG, "no output buffer given");
    double bh[3];
    FCB_TRY(box_to_host(box, bh));
    FCB_TRY(check_cutoff(bh));
    for (int d = 0; d < 3; ++d)
        if (!(r_cut < bh[d])) return set_error(FCB_ERR_CUTOFF, "Cutoff larger than L/2 (r_cut must be < box length)");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 3 * N;
    double *d_pos, *d_box, *d_m;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    FCB_TRY(lj_pair_tables(h, d_pos, N, d_box, sigma, eps, r_cut, s));
    AssemblyOut out;
    const bool host64 = psi_out && !is_device_ptr(psi_out);
    const bool host32 = psi32_mw_out && !is_device_ptr(psi32_mw_out);
    if (host64 && host32) {
        FCB_TRY(h->psi_stage.ensure(sizeof(double) * n * n * n));
        FCB_TRY(h->psi_f32.ensure(sizeof(float) * n * n * n));
    } else if (host64) {
        FCB_TRY(h->psi_stage.ensure(sizeof(double) * n * n * n));
    } else if (host32) {
        FCB_TRY(h->psi_f32.ensure(sizeof(float) * n * n * n));
    }
    out.psi64 = psi_out ? (host64 ? h->psi_stage.as<double>() : psi_out) : nullptr;
    out.psi64_weighted = weighted;
    out.psi32 = psi32_mw_out ? (host32 ? h->psi_f32.as<float>() : psi32_mw_out) : nullptr;
    FCB_TRY(ifc3_dense_write(h, N, tol, d_m, out, s));
    if (host64) FCB_CUDA(cudaMemcpyAsync(psi_out, out.psi64, sizeof(double) * n * n * n, cudaMemcpyDeviceToHost, s));
    if (host32)
        FCB_CUDA(cudaMemcpyAsync(psi32_mw_out, out.psi32, sizeof(float) * n * n * n, cudaMemcpyDeviceToHost, s));
    if (host64 || host32 || !is_device_ptr(pos) || !is_device_ptr(box) || (masses && !is_device_ptr(masses)))
        return check_status(h, s);
    return FCB_OK;
}

int fcb200_mass_weight3(fcb200_handle h, double* psi, const double* masses, int64_t N, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (!psi || !masses) return set_error(FCB_ERR_ARG, "psi and masses must not be NULL");
    if (N < 1) return set_error(FCB_ERR_ARG, "n_atoms must be >= 1");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 3 * N;
    double* d_m;
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    const bool host = !is_device_ptr(psi);
    double* d_psi = psi;
    if (host) {
        FCB_TRY(h->psi_stage.ensure(sizeof(double) * n * n * n));
        d_psi = h->psi_stage.as<double>();
        FCB_CUDA(cudaMemcpyAsync(d_psi, psi, sizeof(double) * n * n * n, cudaMemcpyHostToDevice, s));
    }
    FCB_TRY(mass_weight3_launch(d_psi, d_m, N, s));
    if (host) {
        FCB_CUDA(cudaMemcpyAsync(psi, d_psi, sizeof(double) * n * n * n, cudaMemcpyDeviceToHost, s));
        return check_status(h, s);
    }
    return FCB_OK;
}

int fcb200_second_order_lj(fcb200_handle h, const double* pos, int64_t N, const double* box, double sigma,
                           double eps, double r_cut, double tol, const double* masses, double* ifc2_out,
                           void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    FCB_TRY(validate_lj(pos, N, box, r_cut, masses, false));
    if (!ifc2_out) return set_error(FCB_ERR_ARG, "ifc2_out must not be NULL");
    double bh[3];
    FCB_TRY(box_to_host(box, bh));
    FCB_TRY(check_cutoff(bh));
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 3 * N;
    double *d_pos, *d_box, *d_m, *d_out;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    FCB_TRY(device_view(h->ifc2, (const double*)ifc2_out, n * n, false, s, &d_out));
    FCB_TRY(lj_second_order_launch(h, d_pos, N, d_box, sigma, eps, r_cut, tol, d_m, d_out, s));
    if (d_out != ifc2_out) {
        FCB_CUDA(cudaMemcpyAsync(ifc2_out, d_out, sizeof(double) * n * n, cudaMemcpyDeviceToHost, s));
        return check_status(h, s);
    }
    return FCB_OK;
}

static int validate_sw(const double* pos, int64_t N, const double* box, double r_cut) {
    if (pos == nullptr || box == nullptr) return set_error(FCB_ERR_ARG, "pos and box must not be NULL");
    if (N < 1) return set_error(FCB_ERR_ARG, "n_atoms must be >= 1");
    if (N > 4096) return set_error(FCB_ERR_ARG, "n_atoms > 4096 (dense n³ tensor would exceed device memory)");
    if (!(r_cut > 0.0)) return set_error(FCB_ERR_ARG, "r_cut must be positive");
    if (!(r_cut <= sw_potential_cutoff()))
        return set_error(FCB_ERR_CUTOFF, "For AutoDiff SW silicon force constant cutoff must be less than potential cutoff");
    return FCB_OK;
}

int fcb200_third_order_sw(fcb200_handle h, const double* pos, int64_t N, const double* box, double r_cut, double tol,
                          const double* cos0, const double* masses, double* psi_out, float* psi32_mw_out, int flags,
                          void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    FCB_TRY(validate_sw(pos, N, box, r_cut));
    const bool weighted = (flags & FCB_PSI_MASS_WEIGHTED) != 0;
    if ((weighted || psi32_mw_out) && !masses) return set_error(FCB_ERR_ARG, "masses are required for mass weighting");
    if (!psi_out && !psi32_mw_out) return set_error(FCB_ERR_ARG, "no output buffer given");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 3 * N;
    double *d_pos, *d_box, *d_m;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    const bool host64 = psi_out && !is_device_ptr(psi_out);
    const bool host32 = psi32_mw_out && !is_device_ptr(psi32_mw_out);
    if (host64) FCB_TRY(h->psi_stage.ensure(sizeof(double) * n * n * n));
    if (host32) FCB_TRY(h->psi_f32.ensure(sizeof(float) * n * n * n));
    AssemblyOut out;
    out.psi64 = psi_out ? (host64 ? h->psi_stage.as<double>() : psi_out) : nullptr;
    out.psi64_weighted = weighted;
    out.psi32 = psi32_mw_out ? (host32 ? h->psi_f32.as<float>() : psi32_mw_out) : nullptr;
    FCB_TRY(sw_third_order_launch(h, d_pos, N, d_box, r_cut, cos0, tol, d_m, out, s));
    if (host64) FCB_CUDA(cudaMemcpyAsync(psi_out, out.psi64, sizeof(double) * n * n * n, cudaMemcpyDeviceToHost, s));
    if (host32)
        FCB_CUDA(cudaMemcpyAsync(psi32_mw_out, out.psi32, sizeof(float) * n * n * n, cudaMemcpyDeviceToHost, s));
    return check_status(h, s);
}

int fcb200_second_order_sw(fcb200_handle h, const double* pos, int64_t N, const double* box, double r_cut,
                           double tol, const double* cos0, const double* masses, double* ifc2_out, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    FCB_TRY(validate_sw(pos, N, box, r_cut));
    if (!ifc2_out) return set_error(FCB_ERR_ARG, "ifc2_out must not be NULL");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 3 * N;
    double *d_pos, *d_box, *d_m, *d_out;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    FCB_TRY(device_view(h->ifc2, (const double*)ifc2_out, n * n, false, s, &d_out));
    FCB_TRY(sw_second_order_launch(h, d_pos, N, d_box, r_cut, cos0, tol, d_m, d_out, s));
    if (d_out != ifc2_out)
        FCB_CUDA(cudaMemcpyAsync(ifc2_out, d_out, sizeof(double) * n * n, cudaMemcpyDeviceToHost, s));
    return check_status(h, s);
}

static int mcc3_ranges_ok(int64_t n, int64_t a, int64_t b) { return 0 <= a && a < b && b <= n; }

int fcb200_mcc3(fcb200_handle h, const float* psi, const float* phi, int64_t n, int64_t n_lo, int64_t n_hi,
                int64_t m_lo, int64_t m_hi, int64_t l_lo, int64_t l_hi, int precision, float* k3_out,
                void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (!psi || !phi || !k3_out) return set_error(FCB_ERR_ARG, "psi, phi and k3_out must not be NULL");
    if (n < 1) return set_error(FCB_ERR_ARG, "n must be >= 1");
    if (!mcc3_ranges_ok(n, n_lo, n_hi) || !mcc3_ranges_ok(n, m_lo, m_hi) || !mcc3_ranges_ok(n, l_lo, l_hi))
        return set_error(FCB_ERR_ARG, "mode window outside [0, n)");
    FCB_TRY(check_precision(precision));
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *d_psi, *d_phi, *d_k3;
    FCB_TRY(device_view(h->psi_f32, psi, (size_t)(n * n * n), true, s, &d_psi));
    FCB_TRY(device_view(h->phi_f32, phi, (size_t)(n * n), true, s, &d_phi));
    const size_t k3n = (size_t)((n_hi - n_lo) * (m_hi - m_lo) * (l_hi - l_lo));
    FCB_TRY(device_view(h->k3_stage[0], (const float*)k3_out, k3n, false, s, &d_k3));
    Mcc3Operand op;
    FCB_TRY(psi_operand_from_f32(h, precision, d_psi, n, s, &op));
    FCB_TRY(run_mcc3(h, precision, op, d_phi, n, n_lo, n_hi, m_lo, m_hi, l_lo, l_hi, d_k3, s));
    const bool host_io = d_k3 != k3_out || d_psi != psi || d_phi != phi;
    if (d_k3 != k3_out) FCB_CUDA(cudaMemcpyAsync(k3_out, d_k3, sizeof(float) * k3n, cudaMemcpyDeviceToHost, s));
    if (host_io) return check_status(h, s);
    return FCB_OK;
}

int fcb200_mcc3_blocked(fcb200_handle h, const float* psi, const float* phi, int64_t n, int64_t block_size,
                        int precision, float* k3_out, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (!psi || !phi || !k3_out) return set_error(FCB_ERR_ARG, "psi, phi and k3_out must not be NULL");
    if (n < 1) return set_error(FCB_ERR_ARG, "n must be >= 1");
    if (block_size <= 0 || n % block_size != 0)
        return set_error(FCB_ERR_BLOCK, "size(phi,1) must be a multiple of block_size (mcc.jl:91)");
    FCB_TRY(check_precision(precision));
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *d_psi, *d_phi;
    FCB_TRY(device_view(h->psi_f32, psi, (size_t)(n * n * n), true, s, &d_psi));
    FCB_TRY(device_view(h->phi_f32, phi, (size_t)(n * n), true, s, &d_phi));
    Mcc3Operand op;
    FCB_TRY(psi_operand_from_f32(h, precision, d_psi, n, s, &op));
    const bool host_out = !is_device_ptr(k3_out);
    const int64_t slab = n * n * block_size;  // floats per slab of the last mode axis
    if (!host_out) {
        FCB_TRY(run_mcc3(h, precision, op, d_phi, n, 0, n, 0, n, 0, n, k3_out, s));
    } else {
        // P1 and P2 once, then P3 slab by slab; each slab is copied back on the
        // aux stream while the next one computes.
        FCB_TRY(h->k3_stage[0].ensure(sizeof(float) * slab));
        FCB_TRY(h->k3_stage[1].ensure(sizeof(float) * slab));
        const int64_t nb = n / block_size;
        for (int64_t b = 0; b < nb; ++b) {
            const int slot = (int)(b & 1);
            if (b >= 2) FCB_CUDA(cudaStreamWaitEvent(s, h->ev[slot], 0));  // slot's previous copy done
            float* d_slab = h->k3_stage[slot].as<float>();
            if (b == 0) {
                FCB_TRY(run_mcc3(h, precision, op, d_phi, n, 0, n, 0, n, 0, block_size, d_slab, s));
            } else {
                // Only P3 for the remaining slabs: U2 is already resident.
                const int64_t l0 = b * block_size;
                if (precision == FCB_MCC3_FP32) {
                    ModeProduct p3{n * n, n, block_size, n, n, n * n, n * n, n * n};
                    FCB_TRY(mode_product_f32(h->u2_f32.as<float>(), d_phi + n * l0, d_slab, p3, s));
                } else {
                    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
                    const int64_t np = pad_for(kind, n);
                    const size_t esz = esz_of(kind);
                    ModeProduct p3{n * n, n, block_size, np, np, n * n, n * n, n * n};
                    FCB_TRY(mode_product_tc(h, kind, h->u2_hi.p, h->u2_lo.p,
                                            static_cast<uint8_t*>(h->phi_hi.p) + esz * np * l0,
                                            static_cast<uint8_t*>(h->phi_lo.p) + esz * np * l0, d_slab, nullptr, 0,
                                            p3, s));
                }
            }
            FCB_CUDA(cudaEventRecord(h->ev[2], s));
            FCB_CUDA(cudaStreamWaitEvent(h->aux_stream, h->ev[2], 0));
            FCB_CUDA(cudaMemcpyAsync(k3_out + b * slab, d_slab, sizeof(float) * slab, cudaMemcpyDeviceToHost,
                                     h->aux_stream));
            FCB_CUDA(cudaEventRecord(h->ev[slot], h->aux_stream));
        }
        FCB_CUDA(cudaStreamSynchronize(h->aux_stream));
    }
    if (host_out || d_psi != psi || d_phi != phi) return check_status(h, s);
    return FCB_OK;
}

}  // extern "C"

namespace fcb {
namespace {
// Snapshot driver shared by the LJ and SW entry points: `assemble` writes Ψ
// (optional FP64) and the operand of the chosen precision in one pass, then the
// three mode products run.
template <class Assemble>
int snapshot_run(fcb200_context* h, int64_t N, const float* phi, int64_t mode_lo, int64_t mode_hi, int precision,
                 double* psi_out, float* k3_out, cudaStream_t s, bool host_inputs, Assemble assemble,
                 bool packed = false) {
    const int64_t n = 3 * N;
    float* d_phi;
    FCB_TRY(device_view(h->phi_f32, phi, (size_t)(n * n), true, s, &d_phi));
    for (bool& m : h->marked) m = false;
    phase_mark(h, s, 0);
    const bool host64 = psi_out && !is_device_ptr(psi_out);
    if (host64) FCB_TRY(h->psi_stage.ensure(sizeof(double) * n * n * n));
    AssemblyOut out;
    out.psi64 = psi_out ? (host64 ? h->psi_stage.as<double>() : psi_out) : nullptr;
    Mcc3Operand op;
    if (precision == FCB_MCC3_FP32) {
        FCB_TRY(h->psi_f32.ensure(sizeof(float) * n * n * n));
        out.psi32 = h->psi_f32.as<float>();
        op.f32 = out.psi32;
    } else {
        const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
        const int64_t np = pad_for(kind, n);
        FCB_TRY(h->psi_hi.ensure((size_t)esz_of(kind) * np * n * n));
        FCB_TRY(h->psi_lo.ensure((size_t)esz_of(kind) * np * n * n));
        out.split_hi = h->psi_hi.p;
        out.split_lo = h->psi_lo.p;
        out.split_kind = kind;
        out.n_pad = np;
        op.hi = out.split_hi;
        op.lo = out.split_lo;
    }
    FCB_TRY(assemble(out));  // marks 1 (after the pair/triplet tables) itself
    phase_mark(h, s, 2);
    if (precision == FCB_MCC3_FP32) phase_mark(h, s, 3);  // no φ split phase
    const int64_t M = mode_hi - mode_lo;
    const int64_t k3n = packed ? packed_k3_count(M) : M * M * M;
    float* d_k3;
    FCB_TRY(device_view(h->k3_stage[0], (const float*)k3_out, (size_t)k3n, false, s, &d_k3));
    float* d_full = d_k3;
    if (packed) {  // the full K3 into scratch, then its unique entries
        FCB_TRY(h->k3_full.ensure(sizeof(float) * (size_t)(M * M * M)));
        d_full = h->k3_full.as<float>();
    }
    FCB_TRY(run_mcc3(h, precision, op, d_phi, n, mode_lo, mode_hi, mode_lo, mode_hi, mode_lo, mode_hi, d_full, s,
                     true));
    if (packed) FCB_TRY(pack_k3_launch(d_full, M, d_k3, s));
    bool host = host_inputs || d_phi != phi;
    if (host64) {
        FCB_CUDA(cudaMemcpyAsync(psi_out, out.psi64, sizeof(double) * n * n * n, cudaMemcpyDeviceToHost, s));
        host = true;
    }
    if (d_k3 != k3_out) {
        FCB_CUDA(cudaMemcpyAsync(k3_out, d_k3, sizeof(float) * k3n, cudaMemcpyDeviceToHost, s));
        host = true;
    }
    if (host) return check_status(h, s);
    return FCB_OK;
}

// φ in the split layout of the tensor-core products.
int split_phi(fcb200_context* h, int kind, const float* d_phi, int64_t n, cudaStream_t s) {
    const int64_t np = pad_for(kind, n);
    const size_t esz = esz_of(kind);
    FCB_TRY(h->phi_hi.ensure(esz * np * n));
    FCB_TRY(h->phi_lo.ensure(esz * np * n));
    return split_operand(d_phi, n, n, n, h->phi_hi.p, h->phi_lo.p, np, kind, s);
}

// Coefficient tables, sparse P1 and the symmetric P2/P3 (phase marks 3..5; the
// caller splits φ before and marks 6 after).  after_p1() is called once P1 is
// enqueued and before P2.
template <class AfterP1>
int sparse_products(fcb200_context* h, int64_t N, int64_t mode_lo, int64_t M, int kind, int cap, const int* d_nb,
                    const int* d_count, const int* d_self, double tol, const double* d_m, const float* d_phi,
                    float* d_k3, cudaStream_t s, AfterP1 after_p1) {
    const int64_t n = 3 * N;
    const int64_t np = pad_for(kind, n);
    const size_t esz = esz_of(kind);
    FCB_TRY(h->sp_coef.ensure(sizeof(float) * (size_t)N * 27 * 3 * cap));
    FCB_TRY(lj_sparse_coefs(h, N, tol, d_m, d_nb, d_count, d_self, cap, h->sp_coef.as<float>(), s));
    phase_mark(h, s, 3);
    FCB_TRY(h->u1_hi.ensure(esz * np * n * M));
    FCB_TRY(h->u1_lo.ensure(esz * np * n * M));
    FCB_TRY(sparse_p1_launch(h, kind, N, cap, d_nb, d_count, d_self, h->sp_coef.as<float>(), d_phi, np, mode_lo, M,
                             h->u1_hi.p, h->u1_lo.p, s));
    phase_mark(h, s, 4);
    FCB_TRY(after_p1());
    FCB_TRY(h->u2_hi.ensure(esz * np * M * M));
    FCB_TRY(h->u2_lo.ensure(esz * np * M * M));
    auto plane = [&](const Buf& b, int64_t mode) {
        return static_cast<const void*>(static_cast<const uint8_t*>(b.p) + esz * np * mode);
    };
    // Ψ is symmetric in all three indices: U2[k,p,q] = U2[k,q,p] and
    // K3[p,q,s] = K3[p,s,q], so P2 and P3 compute one triangle of tiles.
    ModeProduct p2{n * M, n, M, np, np, n, np, np * M};
    p2.sym = sym_ok(p2);
    FCB_TRY(mode_product_tc(h, kind, h->u1_hi.p, h->u1_lo.p, plane(h->phi_hi, mode_lo), plane(h->phi_lo, mode_lo),
                            h->u2_hi.p, h->u2_lo.p, kind, p2, s));
    phase_mark(h, s, 5);
    ModeProduct p3{M * M, n, M, np, np, M * M, M * M, M * M};
    ModeProduct p3s{M * M, n, M, np, np, M, M, M * M};
    p3s.sym = true;
    if (sym_ok(p3s)) p3 = p3s;
    FCB_TRY(mode_product_tc(h, kind, h->u2_hi.p, h->u2_lo.p, plane(h->phi_hi, mode_lo), plane(h->phi_lo, mode_lo),
                            d_k3, nullptr, 0, p3, s));
    return FCB_OK;
}

// Compact form of the sparse products: coefficient tables, the compact first
// product (U1c and the per-atom φ rows), the grouped second product
// (U2[p + Mp·k + Mp·n·q], one B per atom, symmetric in (p, q)) and the third
// product reading U2 MN-major (phase marks 3..5; the caller splits φ before and
// marks 6 after).  hook() is called before the first product: the FP64 Ψ
// writer it starts shares the SMs with the first product (CUDA cores, light
// on DRAM) and then with the two tensor-core products.
template <class Hook>
int compact_products(fcb200_context* h, int64_t N, int64_t mode_lo, int64_t M, int kind, int cap, const int* d_nb,
                     const int* d_count, const int* d_self, double tol, const double* d_m, const float* d_phi,
                     float* d_k3, cudaStream_t s, Hook hook, bool packed = false) {
    const int64_t n = 3 * N;
    const int64_t np = pad_for(kind, n);
    const int64_t Mp = compact_Mp(M), Kc = compact_Kc(cap);
    const size_t esz = esz_of(kind);
    FCB_TRY(hook());
    FCB_TRY(h->sp_coef.ensure(sizeof(float) * (size_t)N * 27 * 3 * cap));
    FCB_TRY(lj_sparse_coefs(h, N, tol, d_m, d_nb, d_count, d_self, cap, h->sp_coef.as<float>(), s));
    phase_mark(h, s, 3);
    FCB_TRY(h->u1_hi.ensure(esz * Mp * n * Kc));
    FCB_TRY(h->u1_lo.ensure(esz * Mp * n * Kc));
    FCB_TRY(h->phik_hi.ensure(esz * N * M * Kc));
    FCB_TRY(h->phik_lo.ensure(esz * N * M * Kc));
    FCB_TRY(sparse_p1c_launch(kind, N, cap, d_nb, d_count, d_self, h->sp_coef.as<float>(), d_phi, mode_lo, M, Mp, Kc,
                              h->u1_hi.p, h->u1_lo.p, h->phik_hi.p, h->phik_lo.p, s));
    phase_mark(h, s, 4);
    FCB_TRY(h->u2_hi.ensure(esz * Mp * n * M));
    FCB_TRY(h->u2_lo.ensure(esz * Mp * n * M));
    ModeProduct p2{Mp * n, Kc, M, Mp, Kc, Mp, Mp, Mp * n};
    p2.a_mn = true;        // U1c is stored mode-fastest: U1c[p + Mp·(j' + Kc·k)]
    p2.lda_z = Mp * Kc;
    p2.sym_inner = true;
    p2.inner_upper = true;  // U2 tiles with p / 256 <= q / 256 only: all the third product reads
    p2.b_group = 3 * Mp;
    p2.b_group_ld = M;
    FCB_TRY(mode_product_tc(h, kind, h->u1_hi.p, h->u1_lo.p, h->phik_hi.p, h->phik_lo.p, h->u2_hi.p, h->u2_lo.p, kind,
                            p2, s));
    phase_mark(h, s, 5);
    const size_t poff = esz * np * mode_lo;
    ModeProduct p3{Mp * M, n, M, Mp, np, Mp, M, M * M};
    p3.sym_full = true;  // row tiles with p / 256 <= q / 256, K3 stored by its full symmetry
    p3.packed = packed;  // or only its unique entries, packed
    p3.a_mn = true;
    p3.lda_z = Mp * n;
    p3.Fv = M;
    return mode_product_tc(h, kind, h->u2_hi.p, h->u2_lo.p, static_cast<const uint8_t*>(h->phi_hi.p) + poff,
                           static_cast<const uint8_t*>(h->phi_lo.p) + poff, d_k3, nullptr, 0, p3, s);
}

// The compact form where it applies, else the dense-layout sparse form; the
// hook runs once, before the third product or after the first.
// With `packed`, d_k3 receives the unique entries only: written directly by
// the compact third product, else packed from a full K3 in scratch.
template <class Hook>
int sparse_snapshot_products(fcb200_context* h, int64_t N, int64_t mode_lo, int64_t M, int kind, int cap,
                             const int* d_nb, const int* d_count, const int* d_self, double tol, const double* d_m,
                             const float* d_phi, float* d_k3, cudaStream_t s, Hook hook, bool packed = false) {
    if (tc_pair_enabled() && compact_pays(3 * N, M, cap) && sparse_p1c_smem_bytes(cap) <= 227 * 1024)
        return compact_products(h, N, mode_lo, M, kind, cap, d_nb, d_count, d_self, tol, d_m, d_phi, d_k3, s, hook,
                                packed);
    if (!packed)
        return sparse_products(h, N, mode_lo, M, kind, cap, d_nb, d_count, d_self, tol, d_m, d_phi, d_k3, s, hook);
    FCB_TRY(h->k3_full.ensure(sizeof(float) * (size_t)(M * M * M)));
    FCB_TRY(sparse_products(h, N, mode_lo, M, kind, cap, d_nb, d_count, d_self, tol, d_m, d_phi,
                            h->k3_full.as<float>(), s, hook));
    return pack_k3_launch(h->k3_full.as<float>(), M, d_k3, s);
}

// The LJ snapshot with a block-sparse first mode product (split precisions).
// Needs the largest neighbour count on the host to size the coefficient
// tables, so it synchronises the stream once (after the neighbour lists; the
// φ split is already queued behind them), unless the handle has a fixed
// neighbour capacity (then an overflow is reported by the status word).  The
// FP64 Ψ writer (HBM-bound) runs on the aux stream beside the products (from
// the first one on in the compact form, the second and third otherwise), with
// two blocks per SM so that they stay resident beside the pair kernel's CTA
// (one beside the first product's two); the caller's stream waits
// for it before the end (with phase timing on it runs alone instead, before
// the sparse products).  Sets *used = false, having done nothing visible, when
// the neighbourhoods are so large that the sparse form does not pay; the
// caller then runs the dense path.
int snapshot_lj_sparse(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                       double eps, double r_cut, double tol, const double* d_m, const float* phi, int64_t mode_lo,
                       int64_t mode_hi, int precision, double* psi_out, float* k3_out, cudaStream_t s,
                       bool host_inputs, bool* used, bool packed) {
    *used = false;
    const int64_t n = 3 * N, M = mode_hi - mode_lo;
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    float* d_phi;
    FCB_TRY(device_view(h->phi_f32, phi, (size_t)(n * n), true, s, &d_phi));
    for (bool& m : h->marked) m = false;
    phase_mark(h, s, 0);
    FCB_TRY(lj_pair_tables(h, d_pos, N, d_box, sigma, eps, r_cut, s));
    phase_mark(h, s, 1);
    FCB_TRY(h->sp_ints.ensure(sizeof(int) * (size_t)(N * N + 2 * N + 1)));
    int* d_nb = h->sp_ints.as<int>();
    int* d_count = d_nb + N * N;
    int* d_self = d_count + N;
    int* d_max = d_self + N;
    FCB_TRY(lj_neighbour_lists(h, N, d_nb, d_count, d_self, d_max, s));
    const bool read_back = h->fixed_cap <= 0;
    if (read_back) {
        if (!h->h_pinned) FCB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h->h_pinned), 64));
        FCB_CUDA(cudaMemcpyAsync(h->h_pinned, d_max, sizeof(int), cudaMemcpyDeviceToHost, s));
        FCB_CUDA(cudaEventRecord(h->ev[0], s));
    }
    FCB_TRY(split_phi(h, kind, d_phi, n, s));
    const bool host64 = psi_out && !is_device_ptr(psi_out);
    double* d_psi64 = psi_out;
    if (host64) {
        FCB_TRY(h->psi_stage.ensure(sizeof(double) * n * n * n));
        d_psi64 = h->psi_stage.as<double>();
    }
    // With phase timing on, the writer runs alone on the caller's stream (full
    // grid, before the sparse products) so that every phase times one kernel.
    const bool serial_writer = psi_out && h->profiling;
    if (serial_writer) {
        AssemblyOut out;
        out.psi64 = d_psi64;
        FCB_TRY(ifc3_dense_write(h, N, tol, d_m, out, s));
    }
    int cap = h->fixed_cap;
    if (read_back) {
        FCB_CUDA(cudaEventSynchronize(h->ev[0]));
        cap = h->h_pinned[0];
    }
    cap = (cap + 3) / 4 * 4;  // table stride: a multiple of 4 floats per component
    // The per-atom tables of the sparse form must fit in shared memory; if they
    // do not, the dense path runs (and writes the FP64 Ψ again).
    if (cap < 1 || sparse_p1_smem_bytes(cap, N) > 200 * 1024) return FCB_OK;
    *used = true;
    phase_mark(h, s, 2);
    const int64_t k3n = packed ? packed_k3_count(M) : M * M * M;
    float* d_k3;
    FCB_TRY(device_view(h->k3_stage[0], (const float*)k3_out, (size_t)k3n, false, s, &d_k3));
    bool writer = false;
    auto launch_writer = [&]() -> int {
        if (!psi_out || serial_writer) return FCB_OK;
        FCB_CUDA(cudaEventRecord(h->ev[1], s));
        FCB_CUDA(cudaStreamWaitEvent(h->aux_stream, h->ev[1], 0));
        AssemblyOut out;
        out.psi64 = d_psi64;
        FCB_TRY(ifc3_dense_write(h, N, tol, d_m, out, h->aux_stream, 2));
        FCB_CUDA(cudaEventRecord(h->ev[3], h->aux_stream));
        writer = true;
        return FCB_OK;
    };
    const int rc = sparse_snapshot_products(h, N, mode_lo, M, kind, cap, d_nb, d_count, d_self, tol, d_m, d_phi,
                                            d_k3, s, launch_writer, packed);
    if (writer) FCB_CUDA(cudaStreamWaitEvent(s, h->ev[3], 0));
    FCB_TRY(rc);
    phase_mark(h, s, 6);
    bool host = host_inputs || d_phi != phi;
    if (host64) {
        FCB_CUDA(cudaMemcpyAsync(psi_out, d_psi64, sizeof(double) * n * n * n, cudaMemcpyDeviceToHost, s));
        host = true;
    }
    if (d_k3 != k3_out) {
        FCB_CUDA(cudaMemcpyAsync(k3_out, d_k3, sizeof(float) * k3n, cudaMemcpyDeviceToHost, s));
        host = true;
    }
    if (host) return check_status(h, s);
    return FCB_OK;
}
}  // namespace

// Device-pointer-only LJ snapshot without validation or host synchronisation
// (inputs validated when they were added to a batch); safe inside stream capture.
int snapshot_lj_device(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                       double eps, double r_cut, double tol, const double* d_m, const float* d_phi, int64_t mode_lo,
                       int64_t mode_hi, int precision, float* d_k3, cudaStream_t s) {
    return snapshot_run(h, N, d_phi, mode_lo, mode_hi, precision, nullptr, d_k3, s, false,
                        [&](const AssemblyOut& out) {
                            FCB_TRY(lj_pair_tables(h, d_pos, N, d_box, sigma, eps, r_cut, s));
                            phase_mark(h, s, 1);
                            return ifc3_dense_write(h, N, tol, d_m, out, s);
                        });
}

int snapshot_lj_sparse_device(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                              double eps, double r_cut, double tol, const double* d_m, const float* d_phi,
                              int64_t mode_lo, int64_t mode_hi, int precision, int cap, float* d_k3, cudaStream_t s) {
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    for (bool& m : h->marked) m = false;
    phase_mark(h, s, 0);
    FCB_TRY(lj_pair_tables(h, d_pos, N, d_box, sigma, eps, r_cut, s));
    phase_mark(h, s, 1);
    FCB_TRY(h->sp_ints.ensure(sizeof(int) * (size_t)(N * N + 2 * N + 1)));
    int* d_nb = h->sp_ints.as<int>();
    int* d_count = d_nb + N * N;
    int* d_self = d_count + N;
    int* d_max = d_self + N;
    FCB_TRY(lj_neighbour_lists(h, N, d_nb, d_count, d_self, d_max, s));
    FCB_TRY(split_phi(h, kind, d_phi, 3 * N, s));
    phase_mark(h, s, 2);
    FCB_TRY(sparse_snapshot_products(h, N, mode_lo, mode_hi - mode_lo, kind, cap, d_nb, d_count, d_self, tol, d_m,
                                     d_phi, d_k3, s, [] { return (int)FCB_OK; }));
    phase_mark(h, s, 6);
    return FCB_OK;
}
}  // namespace fcb

extern "C" {

int fcb200_snapshot_lj(fcb200_handle h, const double* pos, int64_t N, const double* box, double sigma, double eps,
                       double r_cut, double tol, const double* masses, const float* phi, int64_t mode_lo,
                       int64_t mode_hi, int precision, double* psi_out, float* k3_out, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    FCB_TRY(validate_lj(pos, N, box, r_cut, masses, true));
    if (!phi || !k3_out) return set_error(FCB_ERR_ARG, "phi and k3_out must not be NULL");
    const int64_t n = 3 * N;
    if (!mcc3_ranges_ok(n, mode_lo, mode_hi)) return set_error(FCB_ERR_ARG, "mode window outside [0, n)");
    const bool force_dense = (precision & FCB_MCC3_FORCE_DENSE) != 0;
    const bool packed = (precision & FCB_K3_PACKED) != 0;
    precision &= ~(FCB_MCC3_FORCE_DENSE | FCB_K3_PACKED);
    FCB_TRY(check_precision(precision));
    double bh[3];
    FCB_TRY(box_to_host(box, bh));
    FCB_TRY(check_cutoff(bh));
    for (int d = 0; d < 3; ++d)
        if (!(r_cut < bh[d])) return set_error(FCB_ERR_CUTOFF, "Cutoff larger than L/2 (r_cut must be < box length)");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double *d_pos, *d_box, *d_m;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    if (precision != FCB_MCC3_FP32 && !force_dense) {
        bool used = false;
        FCB_TRY(snapshot_lj_sparse(h, d_pos, N, d_box, sigma, eps, r_cut, tol, d_m, phi, mode_lo, mode_hi, precision,
                                   psi_out, k3_out, s, d_pos != pos, &used, packed));
        if (used) return FCB_OK;
    }
    return snapshot_run(
        h, N, phi, mode_lo, mode_hi, precision, psi_out, k3_out, s, d_pos != pos,
        [&](const AssemblyOut& out) {
            FCB_TRY(lj_pair_tables(h, d_pos, N, d_box, sigma, eps, r_cut, s));
            phase_mark(h, s, 1);
            return ifc3_dense_write(h, N, tol, d_m, out, s);
        },
        packed);
}

int fcb200_mcc3_adjoint_lj(fcb200_handle h, const double* pos, int64_t N, const double* box, double sigma,
                           double eps, double r_cut, const double* masses, const float* phi, int64_t n_modes,
                           const float* W, int precision, double* dpos, double* dsigma, double* deps, double* L_out,
                           void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    FCB_TRY(validate_lj(pos, N, box, r_cut, masses, true));
    if (!phi || !W || !dpos) return set_error(FCB_ERR_ARG, "phi, W and dpos must not be NULL");
    const int64_t n = 3 * N;
    if (n_modes < 1 || n_modes > n) return set_error(FCB_ERR_ARG, "n_modes must be in [1, 3*n_atoms]");
    const bool g64 = precision == FCB_ADJOINT_FP64;
    if (!g64) FCB_TRY(check_precision(precision));
    double bh[3];
    FCB_TRY(box_to_host(box, bh));
    FCB_TRY(check_cutoff(bh));
    for (int d = 0; d < 3; ++d)
        if (!(r_cut < bh[d])) return set_error(FCB_ERR_CUTOFF, "Cutoff larger than L/2 (r_cut must be < box length)");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double *d_pos, *d_box, *d_m, *d_dpos;
    float *d_phi, *d_W;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    FCB_TRY(device_view(h->phi_f32, phi, (size_t)(n * n), true, s, &d_phi));
    FCB_TRY(device_view(h->adj_w32, W, (size_t)(n_modes * n_modes * n_modes), true, s, &d_W));
    FCB_TRY(device_view(h->adj_dpos, (const double*)dpos, (size_t)(3 * N), false, s, &d_dpos));
    FCB_TRY(h->adj_G.ensure((g64 ? sizeof(double) : sizeof(float)) * (size_t)(n * n * n)));
    FCB_TRY(h->adj_scal.ensure(sizeof(double) * 4));
    FCB_TRY(adjoint_g(h, precision, d_W, n_modes, d_phi, n, h->adj_G.p, s));
    FCB_TRY(lj_adjoint_pairs(h, d_pos, N, d_box, sigma, eps, r_cut, d_m, h->adj_G.p, g64, d_dpos,
                             h->adj_scal.as<double>(), s));
    double sc[3];
    FCB_CUDA(cudaMemcpyAsync(sc, h->adj_scal.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (d_dpos != dpos) FCB_CUDA(cudaMemcpyAsync(dpos, d_dpos, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s));
    FCB_TRY(check_status(h, s));
    if (dsigma) *dsigma = sc[0];
    if (deps) *deps = sc[1];
    if (L_out) *L_out = sc[2];
    return FCB_OK;
}

int fcb200_snapshot_sw(fcb200_handle h, const double* pos, int64_t N, const double* box, double r_cut, double tol,
                       const double* cos0, const double* masses, const float* phi, int64_t mode_lo, int64_t mode_hi,
                       int precision, double* psi_out, float* k3_out, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    FCB_TRY(validate_sw(pos, N, box, r_cut));
    if (!masses) return set_error(FCB_ERR_ARG, "masses are required for mass weighting");
    if (!phi || !k3_out) return set_error(FCB_ERR_ARG, "phi and k3_out must not be NULL");
    const int64_t n = 3 * N;
    if (!mcc3_ranges_ok(n, mode_lo, mode_hi)) return set_error(FCB_ERR_ARG, "mode window outside [0, n)");
    const bool packed = (precision & FCB_K3_PACKED) != 0;
    precision &= ~FCB_K3_PACKED;
    FCB_TRY(check_precision(precision));
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double *d_pos, *d_box, *d_m;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->masses, masses, N, true, s, &d_m));
    return snapshot_run(
        h, N, phi, mode_lo, mode_hi, precision, psi_out, k3_out, s, d_pos != pos,
        [&](const AssemblyOut& out) {
            phase_mark(h, s, 1);
            return sw_third_order_launch(h, d_pos, N, d_box, r_cut, cos0, tol, d_m, out, s);
        },
        packed);
}

// ---------------------------------------------------------------------------
// Finite-difference force constants (third_order_FD.jl, second_order_FD.jl).

static int fd_common(fcb200_handle h, const double* pos, int64_t N, const double* box, double step) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (!pos || !box) return set_error(FCB_ERR_ARG, "pos and box must not be NULL");
    if (N < 1 || N > 4096) return set_error(FCB_ERR_ARG, "n_atoms must be in [1, 4096]");
    if (!(step > 0.0)) return set_error(FCB_ERR_ARG, "the finite-difference step must be positive");
    return FCB_OK;
}

static int fd_third(fcb200_handle h, int kind, const double* pos, int64_t N, const double* box, double sigma,
                    double eps, double r_cut, const int64_t* elems, int64_t m, double step, double* out,
                    void* stream) {
    FCB_TRY(fd_common(h, pos, N, box, step));
    if (m < 0 || (m > 0 && (!elems || !out))) return set_error(FCB_ERR_ARG, "elems and out must hold n_elems entries");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The reference asserts the index ranges (third_order_FD.jl:50-51): check them here.
    std::vector<int64_t> he((size_t)(6 * m));
    if (m > 0) FCB_CUDA(cudaMemcpy(he.data(), elems, sizeof(int64_t) * 6 * m, cudaMemcpyDefault));
    for (int64_t e = 0; e < m; ++e)
        for (int t = 0; t < 3; ++t) {
            if (he[6 * e + 2 * t] < 0 || he[6 * e + 2 * t] >= N)
                return set_error(FCB_ERR_ARG, "Atom indexes out of range, must be in 0:" + std::to_string(N - 1));
            if (he[6 * e + 2 * t + 1] < 0 || he[6 * e + 2 * t + 1] > 2)
                return set_error(FCB_ERR_ARG, "Cartesian indices must be 0, 1, or 2");
        }
    if (m == 0) return FCB_OK;
    double *d_pos, *d_box, *d_out;
    int64_t* d_el;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->fd_elems, elems, (size_t)(6 * m), true, s, &d_el));
    FCB_TRY(device_view(h->fd_out, (const double*)out, (size_t)m, false, s, &d_out));
    FCB_TRY(fd_third_order_launch(d_pos, d_box, N, kind, sigma, eps, r_cut, d_el, m, step, d_out, s));
    if (d_out != out) {
        FCB_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        return check_status(h, s);
    }
    return FCB_OK;
}

static int fd_second(fcb200_handle h, int kind, const double* pos, int64_t N, const double* box, double sigma,
                     double eps, double r_cut, double calc_r_cut, double tol, double step, double* ifc2_out,
                     void* stream) {
    FCB_TRY(fd_common(h, pos, N, box, step));
    if (!ifc2_out) return set_error(FCB_ERR_ARG, "ifc2_out must not be NULL");
    if (!(calc_r_cut > 0.0)) return set_error(FCB_ERR_ARG, "r_cut must be positive");
    cudaSetDevice(h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = 3 * N;
    double *d_pos, *d_box, *d_out;
    FCB_TRY(device_view(h->pos, pos, 3 * N, true, s, &d_pos));
    FCB_TRY(device_view(h->box, box, 3, true, s, &d_box));
    FCB_TRY(device_view(h->ifc2, (const double*)ifc2_out, (size_t)(n * n), false, s, &d_out));
    FCB_TRY(fd_second_order_launch(d_pos, d_box, N, kind, sigma, eps, r_cut, calc_r_cut, tol, step, d_out,
                                   h->d_status, s));
    if (d_out != ifc2_out)
        FCB_CUDA(cudaMemcpyAsync(ifc2_out, d_out, sizeof(double) * n * n, cudaMemcpyDeviceToHost, s));
    return check_status(h, s);
}

int fcb200_fd_third_order_lj(fcb200_handle h, const double* pos, int64_t N, const double* box, double sigma,
                             double eps, double r_cut, const int64_t* elems, int64_t n_elems, double step,
                             double* out, void* stream) {
    if (!(r_cut > 0.0)) return set_error(FCB_ERR_ARG, "r_cut must be positive");
    return fd_third(h, 0, pos, N, box, sigma, eps, r_cut, elems, n_elems, step, out, stream);
}

int fcb200_fd_third_order_sw(fcb200_handle h, const double* pos, int64_t N, const double* box, const int64_t* elems,
                             int64_t n_elems, double step, double* out, void* stream) {
    return fd_third(h, 1, pos, N, box, 0.0, 0.0, 0.0, elems, n_elems, step, out, stream);
}

int fcb200_fd_second_order_lj(fcb200_handle h, const double* pos, int64_t N, const double* box, double sigma,
                              double eps, double r_cut, double calc_r_cut, double tol, double step, double* ifc2_out,
                              void* stream) {
    if (!(r_cut > 0.0)) return set_error(FCB_ERR_ARG, "r_cut must be positive");
    return fd_second(h, 0, pos, N, box, sigma, eps, r_cut, calc_r_cut, tol, step, ifc2_out, stream);
}

int fcb200_fd_second_order_sw(fcb200_handle h, const double* pos, int64_t N, const double* box, double calc_r_cut,
                              double tol, double step, double* ifc2_out, void* stream) {
    return fd_second(h, 1, pos, N, box, 0.0, 0.0, 0.0, calc_r_cut, tol, step, ifc2_out, stream);
}

}  // extern "C"
