// Internal declarations shared by the fcb200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <string>
#include <unordered_map>

#include "../../include/fcb200.h"

namespace fcb {

// ---------------------------------------------------------------------------
// Error reporting: each entry point returns a status; the message is kept per
// thread for fcb200_last_error().
// ---------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);

#define FCB_CUDA(call)                                                  \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ::fcb::cuda_error(e_, #call);     \
    } while (0)

#define FCB_TRY(call)                    \
    do {                                 \
        int s_ = (call);                 \
        if (s_ != FCB_OK) return s_;     \
    } while (0)

// Device-side status word codes (written by bounded waits).
enum DeviceStatus : int {
    DEV_OK = 0,
    DEV_TIMEOUT_PRODUCER = 1,
    DEV_TIMEOUT_MMA = 2,
    DEV_TIMEOUT_EPILOGUE = 3,
    DEV_FD_OVERFLOW = 16,  // a finite-difference neighbourhood exceeded its list capacity
    DEV_SPARSE_OVERFLOW = 17,  // a neighbourhood exceeded the sparse tables' capacity
};

// A device buffer cached in a handle and grown on demand.
struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t need);
    void release();
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Split operand: two planes (hi, lo) of the same padded layout.
struct SplitPlanes {
    void* hi = nullptr;
    void* lo = nullptr;
};

}  // namespace fcb

struct fcb200_context {
    int device = 0;
    int sm_count = 0;
    int* d_status = nullptr;        // device status word (bounded-wait failures)
    uint64_t wait_limit_ns = 2000000000ull;  // limit of the tensor-core kernels' mbarrier waits
    int fixed_cap = 0;  // > 0: the sparse snapshot path's neighbour capacity, no host read-back
    int* h_pinned = nullptr;        // small pinned host buffer for counts read back during a call
    // assembly scratch
    fcb::Buf pos, box, masses;      // staged inputs
    fcb::Buf pair_t, pair_flag;     // per ordered pair: 27 values of -ϕ₃ and a within-cut flag
    fcb::Buf self_t;                // per atom: 27 ASR self values
    fcb::Buf psi_stage;             // device copy of Ψ when the caller passes a host buffer
    // mcc3 scratch
    fcb::Buf phi_f32;               // staged φ (FP32)
    fcb::Buf phi_hi, phi_lo;        // split φ (padded, [modes][n_pad])
    fcb::Buf psi_hi, psi_lo;        // split Ψ
    fcb::Buf u1_hi, u1_lo, u2_hi, u2_lo;  // split intermediates
    fcb::Buf u1_f32, u2_f32;        // plain FP32 intermediates
    fcb::Buf psi_f32;               // staged Ψ (FP32) for host inputs
    fcb::Buf k3_stage[2];           // K3 staging slabs (device) for host outputs
    fcb::Buf k3_full;               // full K3 before packing (FCB_K3_PACKED on the dense paths)
    fcb::Buf ifc2;                  // second-order scratch
    // Stillinger-Weber scratch (neighbours, blocks, placements, buckets, ASR rows)
    fcb::Buf sw_ints, sw_nbr_r, sw_pair_off, sw_blk3, sw_blk2, sw_atoms, sw_place;
    fcb::Buf sw_col_off, sw_col_items, sw_cursor, sw_asr_off, sw_asr_items, sw_asr;
    // adjoint scratch
    fcb::Buf adj_phiT, adj_w_hi, adj_w_lo, adj_pairs, adj_G, adj_scal, adj_w32, adj_dpos;
    fcb::Buf adj_w64, adj_phiT64;   // FP64 forms of W and φᵀ (FCB_ADJOINT_FP64)
    // block-sparse P1 of the LJ snapshot: neighbour lists and coefficient tables
    fcb::Buf sp_ints, sp_coef;
    fcb::Buf phik_hi, phik_lo;      // compact sparse form: per-atom φ rows (split)
    // finite differences: staged element list and output
    fcb::Buf fd_elems, fd_out;
    // get_modes: eigensolver handle (cusolverDnHandle_t, opened on first use) and scratch
    void* solver = nullptr;
    fcb::Buf eig_a, eig_w, eig_work;
    // Autotuned mode-tile counts per mode-product shape (shared by a handle and
    // its batch lanes; owned by the top-level handle).
    std::unordered_map<uint64_t, int>* tune = nullptr;
    bool owns_tune = false;
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // Optional per-phase timing of fcb200_snapshot_lj (events on the caller's stream).
    static constexpr int kMarks = 7;
    bool profiling = false;
    bool marked[kMarks] = {};
    cudaEvent_t pev[kMarks] = {};
};

namespace fcb {

bool is_device_ptr(const void* p);

// Releases the eigensolver handle of a context (modes.cu).
void modes_release(fcb200_context* h);

// Key of a mode-product shape in the autotune table.
inline uint64_t tune_key(int kind, int64_t R, int64_t K, int64_t M) {
    return ((uint64_t)kind << 62) ^ ((uint64_t)R << 24) ^ ((uint64_t)K << 12) ^ (uint64_t)M;
}

// Records phase mark i on stream s when profiling is enabled.
inline void phase_mark(fcb200_context* h, cudaStream_t s, int i) {
    if (h->profiling && i < fcb200_context::kMarks) {
        cudaEventRecord(h->pev[i], s);
        h->marked[i] = true;
    }
}

// ---------------------------------------------------------------------------
// LJ assembly (lj_assembly.cu)
// ---------------------------------------------------------------------------
struct AssemblyOut {
    double* psi64 = nullptr;        // n³ FP64 (column-major), may be null
    bool psi64_weighted = false;    // write the mass-weighted value into psi64
    float* psi32 = nullptr;         // n³ FP32 mass weighted (dense, stride n), may be null
    void* split_hi = nullptr;       // split mass-weighted copy, padded stride n_pad
    void* split_lo = nullptr;
    int split_kind = 0;             // 0 none, 1 bf16 planes, 2 tf32 (fp32) planes
    int64_t n_pad = 0;
};

int lj_pair_tables(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box,
                   double sigma, double eps, double r_cut, cudaStream_t s);
// blocks_per_sm caps the grid (grid-stride loop); a small cap leaves room on
// every SM for a kernel that runs beside the writer on another stream.
int ifc3_dense_write(fcb200_context* h, int64_t N, double tol, const double* d_masses,
                     const AssemblyOut& out, cudaStream_t s, int blocks_per_sm = 8);
int mass_weight3_launch(double* d_psi, const double* d_masses, int64_t N, cudaStream_t s);
int lj_pair_tables_raw(double* T, uint8_t* flag, double* S, const double* d_pos, int64_t N, const double* d_box,
                       double sigma, double eps, double r_cut, cudaStream_t s);
int ifc3_dense_write_raw(const double* T, const uint8_t* flag, const double* S, int sm_count, int64_t N, double tol,
                         const double* d_masses, const AssemblyOut& out, cudaStream_t s);
int lj_second_order_launch(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box,
                           double sigma, double eps, double r_cut, double tol,
                           const double* d_masses, double* d_ifc2, cudaStream_t s);

// Stillinger-Weber (sw_assembly.cu).  cos0 = {cosθ₀ of the generated blocks,
// cosθ₀ of the iik block}, NULL for the reference's values.
double sw_potential_cutoff();
int sw_third_order_launch(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double r_cut,
                          const double* cos0, double tol, const double* d_masses, const AssemblyOut& out,
                          cudaStream_t s);
int sw_second_order_launch(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double r_cut,
                           const double* cos0, double tol, const double* d_masses, double* d_ifc2, cudaStream_t s);

// Device-only snapshot (capi.cu), used by the batch engine (batch.cu).
// Block-sparse LJ snapshot without any host synchronisation: `cap` (a multiple
// of 4, at least the largest neighbourhood including the atom itself) is fixed
// by the caller; safe inside stream capture.
int snapshot_lj_sparse_device(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                              double eps, double r_cut, double tol, const double* d_m, const float* d_phi,
                              int64_t mode_lo, int64_t mode_hi, int precision, int cap, float* d_k3, cudaStream_t s);
int snapshot_lj_device(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                       double eps, double r_cut, double tol, const double* d_m, const float* d_phi, int64_t mode_lo,
                       int64_t mode_hi, int precision, float* d_k3, cudaStream_t s);

// Adjoint (adjoint.cu)
// G is FP64 (n³ doubles) for FCB_ADJOINT_FP64, FP32 otherwise.
int adjoint_g(fcb200_context* h, int precision, const float* d_W, int64_t M, const float* d_phi, int64_t n,
              void* d_G, cudaStream_t s);
int lj_adjoint_pairs(fcb200_context* h, const double* d_pos, int64_t N, const double* d_box, double sigma,
                     double eps, double r_cut, const double* d_masses, const void* d_G, bool g64, double* d_dpos,
                     double* d_scal, cudaStream_t s);

// ---------------------------------------------------------------------------
// mcc3 (mcc3.cu, mode_product_simt.cu, mode_product_tc.cu)
// ---------------------------------------------------------------------------
// One mode product  D[r,p] = Σ_a A[a + lda*r] * B[a + ldb*p],  r < R, p < M,
// a < K; D stored at (r % F) + F_pad*(r / F) + ldd*p.
struct ModeProduct {
    int64_t R, K, M;
    int64_t lda, ldb;
    int64_t F, F_pad, ldd;
    // Output symmetric under exchanging the row's outer index (r / F) and the
    // column (e.g. U2[k,p,q] = U2[k,q,p]): tiles whose columns all lie below
    // their rows' outer index are skipped and every computed entry with
    // column > outer index is also stored mirrored.  Needs R = F·M rows.
    bool sym = false;
    // The forms below run on the 2-CTA tensor-core tile only, with R a
    // multiple of 256 and F, F_pad, ldd, Fv and M multiples of 8.
    // Output symmetric under exchanging the row's inner index (r % F) and the
    // column, inside each outer block (U2[k,p,q] = U2[k,q,p] with rows p + F·k):
    // tiles wholly below the diagonal are skipped and tiles wholly above it are
    // also stored transposed.  F a multiple of 256; mode tiles 256 wide.
    bool sym_inner = false;
    // With sym_inner: store the computed tiles only (no transposed copies); the
    // tiles below the (p, q) tile diagonal stay unwritten, for a consumer that
    // reads only tiles with p / 256 <= q / 256 (sym_full).
    bool inner_upper = false;
    // Output symmetric in all three indices (K3 of an assembled IFC3 over equal
    // mode windows): rows r = a + F·b (rows with a >= Fv are padding), columns
    // s, T(x) = x / 256.  Only row tiles with T(a) <= T(b) are computed (every
    // column), and each computed entry is stored at (a,b,s), at (a,s,b) when
    // T(s) < T(a), at (s,a,b) when T(s) > T(b) and at (s,b,a) when
    // T(s) > T(b) > T(a): every entry of the output exactly once.  FP32 output,
    // F a multiple of 256, R = F·M, 256-wide mode tiles.
    bool sym_full = false;
    // With sym_full: store only the entries a <= b <= s, each once, into the
    // packed layout s(s+1)(s+2)/6 + b(b+1)/2 + a (FCB_K3_PACKED) instead of
    // the M³ output.
    bool packed = false;
    // A read MN-major: A[r,a] at (r % F) + lda·a + lda_z·(r / F); F a multiple
    // of 128 and R of F.
    bool a_mn = false;
    int64_t lda_z = 0;
    // Grouped B: rows [g·b_group, (g+1)·b_group) of A use B[a + ldb·(p + b_group_ld·g)]
    // (0 = one B for all rows); b_group a multiple of 256.
    int64_t b_group = 0, b_group_ld = 0;
    // Rows with r % F >= Fv are computed but not stored (0 = F).
    int64_t Fv = 0;
};

int mode_product_f32(const float* A, const float* B, float* D, const ModeProduct& mp,
                     cudaStream_t s);
// Packed symmetry-unique copy of a full M³ K3: packed[s(s+1)(s+2)/6 + q(q+1)/2 + p]
// = K3[p + M(q + M s)] for p <= q <= s (mcc3.cu).
int pack_k3_launch(const float* full, int64_t M, float* packed, cudaStream_t s);
inline int64_t packed_k3_count(int64_t M) { return M * (M + 1) * (M + 2) / 6; }
// FP64 mode product (FP64 tensor cores, mma.sync .f64) and an FP32 → FP64 widening copy (mode_product_f64.cu).
int mode_product_f64(const double* A, const double* B, double* D, const ModeProduct& mp, cudaStream_t s);
int widen_f32_to_f64(const float* src, double* dst, int64_t count, cudaStream_t s);
// Finite-difference IFCs (finite_diff.cu).  kind 0 = LJ, 1 = SW.
int fd_third_order_launch(const double* d_pos, const double* d_box, int64_t N, int kind, double sigma, double eps,
                          double r_cut, const int64_t* d_elems, int64_t m, double h, double* d_out, cudaStream_t s);
int fd_second_order_launch(const double* d_pos, const double* d_box, int64_t N, int kind, double sigma, double eps,
                           double r_cut, double calc_r_cut, double tol, double h, double* d_ifc2, int* d_status,
                           cudaStream_t s);

// Block-sparse first mode product of the LJ snapshot (lj_assembly.cu, sparse_mcc3.cu).
int lj_neighbour_lists(fcb200_context* h, int64_t N, int* d_nb, int* d_count, int* d_self, int* d_max,
                       cudaStream_t s);
int lj_sparse_coefs(fcb200_context* h, int64_t N, double tol, const double* d_masses, const int* d_nb,
                    const int* d_count, const int* d_self, int cap, float* d_coef, cudaStream_t s);
size_t sparse_p1_smem_bytes(int cap, int64_t N);
// Compact first product (sparse_mcc3.cu): U1c[j' + Kc·(p + Mp·k)] and the
// per-atom φ rows φK[j' + Kc·(q + M·K)], split into hi/lo planes of `kind`.
size_t sparse_p1c_smem_bytes(int cap);
int sparse_p1c_launch(int kind, int64_t N, int cap, const int* d_nb, const int* d_count, const int* d_self,
                      const float* d_coef, const float* d_phi, int64_t mode_lo, int64_t M, int64_t Mp, int64_t Kc,
                      void* u1_hi, void* u1_lo, void* pk_hi, void* pk_lo, cudaStream_t s);
// Whether mode products run on the 2-CTA tile (mode_product_tc.cu).
bool tc_pair_enabled();
// Shapes of the compact sparse products: modes padded to whole 256-row blocks,
// neighbourhood rows to a multiple of 16 (the first product stores 16 rows
// of a mode as one 32-byte sector per plane).
inline int64_t compact_Mp(int64_t M) { return (M + 255) / 256 * 256; }
inline int64_t compact_Kc(int cap) { return (3 * (int64_t)cap + 15) / 16 * 16; }
// The compact form pays when its grouped second product and padded third
// product execute at least 10 % fewer tile flops than the dense-K pair.
inline bool compact_pays(int64_t n, int64_t M, int cap) {
    if (M % 8 != 0) return false;
    const double Mp = (double)compact_Mp(M), Kc = (double)compact_Kc(cap);
    const double compact = Mp * n * Kc + Mp * M * n;
    const double dense = (double)n * M * n + (double)M * M * n;
    return compact < 0.9 * dense;
}
int sparse_p1_launch(fcb200_context* h, int kind, int64_t N, int cap, const int* d_nb, const int* d_count,
                     const int* d_self, const float* d_coef, const float* d_phi, int64_t np, int64_t mode_lo,
                     int64_t M, void* u1_hi, void* u1_lo, cudaStream_t s);

// Split operands (hi/lo planes).  kind 1 = bf16, 2 = tf32 (fp32 planes).
// out_kind: 0 = fp32 D (D_hi only), 1 = bf16 split D, 2 = tf32 split D.
int mode_product_tc(fcb200_context* h, int kind, const void* A_hi, const void* A_lo,
                    const void* B_hi, const void* B_lo, void* D_hi, void* D_lo, int out_kind,
                    const ModeProduct& mp, cudaStream_t s);
int split_operand(const float* src, int64_t rows, int64_t cols, int64_t ld_src, void* hi, void* lo,
                  int64_t ld_dst, int kind, cudaStream_t s);

int pad_for(int kind, int64_t n);  // padded leading dimension for a split kind

}  // namespace fcb
