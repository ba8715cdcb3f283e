/*
 * fcb200 — B200-native third-order force constants and modal coupling constants.
 *
 * A C ABI over hand-written sm_100a kernels.  It is the drop-in target for the
 * ForceConstants.jl hot path: dense third-order IFC assembly (LJ analytical and
 * Stillinger-Weber), acoustic-sum-rule self terms, the tolerance cutoff, mass
 * weighting and the `mcc3` modal contraction
 *     K3[n,m,l] = Σ_ijk Ψ[i,j,k] φ[i,n] φ[j,m] φ[k,l].
 *
 * Conventions (all entry points):
 *  - Every function returns an int status (FCB_OK = 0).  No exception or abort
 *    crosses the ABI; fcb200_last_error() returns the message of the calling
 *    thread's last failure.
 *  - Sizes are int64_t.  Arrays are column-major (Julia layout).  Degree of
 *    freedom index = 3*(atom) + component, 0-based here (Julia's 3(a-1)+α).
 *    Ψ[ii,jj,kk] lives at ii + n*(jj + n*kk), n = 3*n_atoms.
 *  - Positions are pos[3*a + x] (Julia's Vector{SVector{3}} flattened).
 *  - Pointers may be host or device memory unless noted; the library detects
 *    which (cudaPointerGetAttributes) and stages host buffers itself.
 *  - `stream` is a cudaStream_t (NULL = the legacy default stream).  Calls with
 *    only device buffers are asynchronous on that stream; calls that read or
 *    write a host buffer synchronise the stream before returning.
 *  - The caller owns every buffer it passes.  A handle owns the library's
 *    scratch (pair tables, split operands, mode-product intermediates) and
 *    caches it between calls.  A handle is not thread-safe; use one per thread.
 */
#ifndef FCB200_H
#define FCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define FCB_OK              0
#define FCB_ERR_ARG         1  /* null pointer, bad size, inconsistent shape              */
#define FCB_ERR_CUTOFF      2  /* r_cut not below the box (third_order_analytical.jl:7)   */
#define FCB_ERR_OOM         3  /* device memory / admission refused                       */
#define FCB_ERR_CUDA        4  /* CUDA runtime or driver error                            */
#define FCB_ERR_TIMEOUT     5  /* a bounded device-side wait gave up (status word set)     */
#define FCB_ERR_UNSUPPORTED 6  /* device is not sm_100 / precision not available          */
#define FCB_ERR_BLOCK       7  /* size(phi,1) % block_size != 0 (mcc.jl:91-92)            */

/* ---- mcc3 precision modes ------------------------------------------------ */
#define FCB_MCC3_FP32       0  /* plain FP32 SIMT mode products (FFMA)                     */
#define FCB_MCC3_BF16X3     1  /* split-BF16 on tcgen05: hi·hi + hi·lo + lo·hi, FP32 acc   */
#define FCB_MCC3_TF32X3     2  /* split-TF32 on tcgen05: hi·hi + hi·lo + lo·hi, FP32 acc   */
/* fcb200_mcc3_adjoint_lj only: G = W ×₁φᵀ ×₂φᵀ ×₃φᵀ formed in FP64 (DMMA)    */
#define FCB_ADJOINT_FP64    3
/* OR into the precision of fcb200_snapshot_lj: run the dense first and second
 * mode products even where the block-sparse form applies.                     */
#define FCB_MCC3_FORCE_DENSE 0x100
/* OR into the precision of fcb200_snapshot_lj / _sw: k3_out receives only the
 * symmetry-unique entries K3[p,q,s], p <= q <= s (K3 of an assembled IFC3 is
 * symmetric in its three indices), p fastest: entry (p,q,s) at
 * s(s+1)(s+2)/6 + q(q+1)/2 + p, M(M+1)(M+2)/6 floats in all (M modes).  The
 * reference computes the full tensor and notes the unique part as a TODO
 * (src/mcc.jl:116-117).                                                        */
#define FCB_K3_PACKED 0x200

/* ---- flags for fcb200_third_order_* -------------------------------------- */
#define FCB_PSI_MASS_WEIGHTED 1 /* write Ψ already divided by sqrt(m_i m_j m_k) into psi_out */

typedef struct fcb200_context* fcb200_handle;

/* Library version (major*10000 + minor*100 + patch). */
int fcb200_version(void);

/* Copies the calling thread's last error message into buf (always terminated).
 * Returns the status code of that error. */
int fcb200_last_error(char* buf, size_t len);

/* Creates a handle bound to CUDA device `device`.  Fails with
 * FCB_ERR_UNSUPPORTED on devices other than compute capability 10.x. */
int fcb200_create(fcb200_handle* out, int device);
int fcb200_destroy(fcb200_handle h);

/* Releases the cached scratch of a handle (kept otherwise until destroy). */
int fcb200_trim(fcb200_handle h);

/* Synchronises `stream` and reports a device-side error recorded by a
 * bounded wait (FCB_ERR_TIMEOUT) since the last check. */
int fcb200_synchronize(fcb200_handle h, void* stream);

/* Limit, in nanoseconds, of every mbarrier wait in the tensor-core kernels of
 * this handle (no counterpart in the reference).  A wait that runs out sets
 * the device status word, the kernel drains the copies and MMAs it issued
 * (those drains always get 2 s), frees its tensor memory and returns, and the
 * next fcb200_synchronize reports FCB_ERR_TIMEOUT; the handle stays usable.
 * limit_ns <= 0 restores the default of 2 s. */
int fcb200_set_wait_limit(fcb200_handle h, int64_t limit_ns);

/* Neighbour capacity of the block-sparse snapshot path (no counterpart in the
 * reference).  cap = 0 (the default): fcb200_snapshot_lj reads the largest
 * neighbour count back to the host once per call (one synchronisation of the
 * stream, after the neighbour lists) and sizes its tables by it.  cap > 0: the
 * tables are sized for `cap` neighbours per atom (rounded up to a multiple of
 * 4), the call does not synchronise (so it can be captured in a CUDA graph
 * after one uncaptured call has sized the handle's scratch), and an atom with
 * more neighbours is reported as FCB_ERR_ARG, K3 invalid (the FP64 Ψ is still
 * written): by the call itself when it synchronises (host positions or host
 * outputs), else by the next fcb200_synchronize.  cap < 0 is FCB_ERR_ARG. */
int fcb200_set_neighbour_capacity(fcb200_handle h, int cap);

/*
 * Dense third-order IFCs of a pair Lennard-Jones system with the analytical
 * calculator.  Replaces
 *   third_order(sys, pot::LJ, AnalyticalCalculator(tol, r_cut))   src/ifc.jl:20-35
 *   third_order!(Ψ, sys, ::PairPotential, ::AnalyticalCalculator)
 *                                        src/analytical/third_order_analytical.jl:4-69
 *   ASR!(ifc3, N, D)                     src/asr.jl:19-40
 *   apply_tols!(Ψ, tol)                  src/helper_funcs.jl:20-27
 * and, fused into the same pass,
 *   mass_weight_third_order!(Ψ, masses)  src/analytical/third_order_analytical.jl:185-214
 *   CuArray{Float32}(Ψ_mw)               README.md:73-75
 *
 * pos       3*n_atoms doubles (Å), box 3 doubles (orthorhombic box lengths).
 * sigma,eps LJ parameters (any consistent units; Ψ is in eps/length³).
 * masses    n_atoms doubles, or NULL (required when psi32_mw_out is given or
 *           flags has FCB_PSI_MASS_WEIGHTED).
 * psi_out   n³ doubles or NULL: Ψ after ASR and tol (mass weighted if flagged).
 * psi32_mw_out  n³ floats or NULL: FP32 copy of the mass-weighted Ψ.
 * Returns FCB_ERR_CUTOFF when r_cut >= a box length (the reference asserts
 * r_cut < L, third_order_analytical.jl:7), FCB_ERR_ARG when both outputs
 * are NULL.
 */
int fcb200_third_order_lj(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                          double sigma, double eps, double r_cut, double tol,
                          const double* masses, double* psi_out, float* psi32_mw_out,
                          int flags, void* stream);

/*
 * In-place mass weighting of a dense third-order IFC tensor: every non-zero
 * Ψ[ii,jj,kk] /= sqrt(m_i*m_j*m_k).  Replaces
 *   mass_weight_third_order!(Ψ, masses)  src/analytical/third_order_analytical.jl:185-214
 */
int fcb200_mass_weight3(fcb200_handle h, double* psi, const double* masses, int64_t n_atoms,
                        void* stream);

/*
 * Dense second-order IFCs (n×n) of an LJ system with the analytical calculator.
 * Replaces second_order(sys, pot::LJ, AnalyticalCalculator)  src/ifc.jl:3-18,
 * second_order!  src/analytical/second_order_analytical.jl:3-42, ASR!(ifc2)
 * src/asr.jl:3-17.  With masses != NULL the result is the dynamical matrix
 * (dynamical_matrix, src/dynmat.jl:5-33).
 */
int fcb200_second_order_lj(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                           double sigma, double eps, double r_cut, double tol,
                           const double* masses, double* ifc2_out, void* stream);

/*
 * Eigen-decomposition of a dynamical matrix on the device.  Replaces
 * get_modes(dynmat, num_rigid_translation = 3)  src/dynmat.jl:123-141:
 * ascending eigenvalues (freqs_sq, length n) and orthonormal eigenvectors
 * (modes, n×n column-major, column c = mode c) of the symmetric n×n FP64
 * matrix (upper triangle used, as Hermitian(A)); the num_rigid eigenvalues
 * nearest zero (stable order of |λ|) are set to 0.  phi32 (nullable) receives
 * the eigenvectors as FP32 — the φ operand of fcb200_mcc3.  modes may be NULL
 * (vectors discarded) or equal to dynmat (in place).  Any pointer may be host or
 * device memory.  Synchronises the stream (the solver's convergence flag is
 * read); a solver that does not converge returns FCB_ERR_CUDA.  Uses
 * libcusolver, opened on first use (FCB_ERR_UNSUPPORTED when absent).
 */
int fcb200_get_modes(fcb200_handle h, const double* dynmat, int64_t n, int num_rigid,
                     double* freqs_sq, double* modes, float* phi32, void* stream);

/*
 * Dense third-order IFCs of Stillinger-Weber silicon (LAMMPS Si.sw parameters,
 * eV and Å), the AutoDiffCalculator path of the reference.  Replaces
 *   third_order(sys, ::StillingerWeberSilicon, AutoDiffCalculator(tol, r_cut))
 *     src/ifc.jl:20-35, src/autodiff/third_order_AD.jl:71-224, src/asr.jl:19-40
 * with analytic derivatives instead of generated AD kernels.  cos0 = {cosθ₀
 * of the blocks the reference takes from its generated kernels (written there
 * as -0.333333333333), cosθ₀ of the iik block (built at run time from the exact
 * -1/3)}; NULL selects exactly those values.  r_cut must not exceed the SW
 * cutoff aσ (third_order_AD.jl:74), else FCB_ERR_CUTOFF.  Outputs as in
 * fcb200_third_order_lj.  Synchronises the stream (it sizes its scratch from
 * the neighbour count).
 */
int fcb200_third_order_sw(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                          double r_cut, double tol, const double* cos0, const double* masses,
                          double* psi_out, float* psi32_mw_out, int flags, void* stream);

/*
 * Dense second-order IFCs of Stillinger-Weber silicon; with masses != NULL the
 * dynamical matrix.  Replaces second_order(sys, ::StillingerWeberSilicon,
 * AutoDiffCalculator) — src/ifc.jl:3-18, src/autodiff/second_order_AD.jl:40-110,
 * src/asr.jl:3-17, src/dynmat.jl:5-33.  cos0 as above (only cos0[0] is used).
 */
int fcb200_second_order_sw(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                           double r_cut, double tol, const double* cos0, const double* masses,
                           double* ifc2_out, void* stream);

/*
 * Third-order modal coupling constants
 *   K3[a,b,c] = Σ_ijk Ψ[i,j,k] φ[i,n_lo+a] φ[j,m_lo+b] φ[k,l_lo+c]
 * for the mode windows [n_lo,n_hi) × [m_lo,m_hi) × [l_lo,l_hi), as three
 * successive mode products.  Replaces
 *   mcc3(Ψ::CuArray{Float32,3}, φ::CuArray{Float32,2})     src/mcc.jl:29-51
 *   mcc3!(Ψ, φ) / mcc3_tens_opt(Ψ, φ)                       src/mcc.jl:11-20, 60-80
 *   mcc3_blocked!(K3, Ψ, φ, ranges)  (one block)            src/mcc.jl:123-134
 * psi    n³ floats (mass-weighted Ψ), phi n×n floats (columns = modes),
 * k3_out (n_hi-n_lo)(m_hi-m_lo)(l_hi-l_lo) floats, column-major.
 * precision is one of FCB_MCC3_*.
 */
int fcb200_mcc3(fcb200_handle h, const float* psi, const float* phi, int64_t n,
                int64_t n_lo, int64_t n_hi, int64_t m_lo, int64_t m_hi, int64_t l_lo, int64_t l_hi,
                int precision, float* k3_out, void* stream);

/*
 * Full K3 computed block-wise with a bounded device footprint.  Replaces
 *   mcc3(Ψ, φ, block_size)   src/mcc.jl:89-120
 * The result (n³ floats) is normally a host buffer, as in the reference; the
 * (n/block_size) slabs of the last mode axis are copied back while the next
 * slab computes.  Fails with FCB_ERR_BLOCK unless n % block_size == 0 and
 * block_size > 0 (mcc.jl:91-92).
 */
int fcb200_mcc3_blocked(fcb200_handle h, const float* psi, const float* phi, int64_t n,
                        int64_t block_size, int precision, float* k3_out, void* stream);

/*
 * One LJ snapshot end to end: dense FP64 IFC3 assembly (+ASR, tol), fused
 * mass weighting into the operand format of the chosen precision, then mcc3
 * over modes [mode_lo, mode_hi) on every axis.  The composition of
 *   third_order (src/ifc.jl:20-35), mass_weight_third_order!
 *   (third_order_analytical.jl:185-214), the Float32 cast (README.md:73-75)
 *   and mcc3 (src/mcc.jl:29-51)
 * without the host round trip.  psi_out (n³ doubles, unweighted) may be NULL;
 * k3_out holds (mode_hi-mode_lo)³ floats.
 * With a split precision the mode products use the block sparsity of the LJ
 * Ψ (non-zeros of the columns of atom K lie in rows of K's neighbourhood) and
 * its symmetry: P1 as a sparse contraction that keeps only the neighbourhood
 * rows, P2 as one GEMM per atom over its neighbours' degrees of freedom
 * (symmetric in its two mode indices), P3 dense over the atoms with symmetric
 * tiles — or, where that does not pay (small cells, mode counts not a multiple
 * of 8), P1 written in the dense layout and symmetric dense P2/P3.  Same K3
 * within the mcc3 tolerance; this form synchronises the stream once (after the
 * neighbour lists), and writes psi_out on a second stream beside the last
 * product.  FCB_MCC3_FORCE_DENSE selects the dense products; FCB_K3_PACKED
 * writes only the symmetry-unique entries of K3 (k3_out then holds
 * M(M+1)(M+2)/6 floats, M = mode_hi - mode_lo).
 */
int fcb200_snapshot_lj(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                       double sigma, double eps, double r_cut, double tol, const double* masses,
                       const float* phi, int64_t mode_lo, int64_t mode_hi, int precision,
                       double* psi_out, float* k3_out, void* stream);

/*
 * One Stillinger-Weber snapshot end to end: SW IFC3 assembly (as
 * fcb200_third_order_sw) with the fused mass-weighted operand, then mcc3 over
 * modes [mode_lo, mode_hi) on every axis.  Same composition as
 * fcb200_snapshot_lj for the reference's AutoDiffCalculator SW path;
 * FCB_K3_PACKED as there.
 */
int fcb200_snapshot_sw(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                       double r_cut, double tol, const double* cos0, const double* masses,
                       const float* phi, int64_t mode_lo, int64_t mode_hi, int precision,
                       double* psi_out, float* k3_out, void* stream);

/*
 * Adjoint of an LJ snapshot (no counterpart in the reference, which has no
 * gradients): for L = Σ_abc W[a,b,c] K3[a,b,c] with K3 over modes [0,n_modes)
 * on every axis (φ frozen), the gradients ∂L/∂positions (dpos, 3*n_atoms
 * doubles), ∂L/∂σ and ∂L/∂ε, and L itself.  G = W ×₁φᵀ ×₂φᵀ ×₃φᵀ is formed by
 * the transposed mode products (precision as for mcc3), then every pair inside
 * the cutoff contracts its recomputed ϕ₃ blocks (third_order_analytical.jl:216-224),
 * their fourth derivatives ϕ₄ (fourth_order_analytical.jl:184-198) and
 * σ-derivatives with G; Ψ and the fourth-order tensor are never stored.  The
 * tolerance cutoff of Ψ is not differentiated.  W is n_modes³ floats,
 * column-major.  precision: FCB_MCC3_FP32 / _BF16X3 / _TF32X3, or
 * FCB_ADJOINT_FP64 (G in double precision: the gradient then carries FP64
 * rounding only).  Synchronises the stream.
 */
int fcb200_mcc3_adjoint_lj(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                           double sigma, double eps, double r_cut, const double* masses,
                           const float* phi, int64_t n_modes, const float* W, int precision,
                           double* dpos, double* dsigma, double* deps, double* L_out, void* stream);

/*
 * Mode-product tile autotuner (no counterpart in the reference).  Times the
 * candidate mode-tile counts of the tensor-core mode product for a full-mode
 * mcc3 of side n (BF16×3 / TF32×3) and keeps the fastest in the handle; with
 * cache_path != NULL the table is read from and written to that JSON file.
 * Later mcc3, snapshot and batch calls of the handle use it.
 */
int fcb200_autotune_mcc3(fcb200_handle h, int64_t n, int precision, const char* cache_path, void* stream);

/*
 * Finite-difference force constants: an independent numerical check of the
 * analytical (LJ) and AD (SW) assemblies.  Replace
 *   third_order_finite_diff_eng(sys, pot, atom_idxs, cartesian_idxs; h)
 *                                   src/finitediff/third_order_FD.jl:43-113
 *   second_order(sys, pot, FiniteDiffCalculator(tol, r_cut; h))
 *                                   src/ifc.jl:3-18, src/finitediff/second_order_FD.jl:3-79
 * with the reference's energy stencils (energy_loop, finitediff_helper.jl:3-64).
 * elems: n_elems rows of 6 int64 (atom, component) pairs (i,α,j,β,k,γ),
 * 0-based; out[e] the stencil value, NaN for the arrangements the reference
 * has no stencil for (i = j != k, j = k != i).  The stencils are the
 * reference's as written: (i,α,j,β,i,γ) displaces only (i,α) and (j,β); (i,α,
 * i,β,i,γ) only (i,α).  Each stencil point sums the energy terms that involve
 * its displaced atoms (the rest cancels because the weights sum to zero).
 * step: the displacement h in Å (the reference's default is 0.04 bohr =
 * 0.021167 Å).  LJ energies use the potential's r_cut; the IFC2 pairs are those
 * within calc_r_cut at the given positions, followed by ASR and apply_tols!(tol).
 * SW: LAMMPS Si.sw parameters with cosθ₀ = -1/3.  FCB_ERR_UNSUPPORTED when more
 * than 128 atoms lie within the SW cutoff of a displaced atom.
 */
int fcb200_fd_third_order_lj(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                             double sigma, double eps, double r_cut, const int64_t* elems,
                             int64_t n_elems, double step, double* out, void* stream);
int fcb200_fd_third_order_sw(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                             const int64_t* elems, int64_t n_elems, double step, double* out,
                             void* stream);
int fcb200_fd_second_order_lj(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                              double sigma, double eps, double r_cut, double calc_r_cut, double tol,
                              double step, double* ifc2_out, void* stream);
int fcb200_fd_second_order_sw(fcb200_handle h, const double* pos, int64_t n_atoms, const double* box,
                              double calc_r_cut, double tol, double step, double* ifc2_out, void* stream);

/*
 * Batches of LJ snapshots (no counterpart in the reference, which runs one
 * snapshot at a time through third_order → mass_weight_third_order! → mcc3,
 * README.md:69-76).  A batch keeps device copies of each snapshot's positions,
 * box, masses and φ; fcb200_batch_run executes all of them: snapshots are
 * admitted into up to 4 parallel lanes by HBM footprint (hbm_budget_bytes of
 * scratch; 0 = 80 % of free memory), the first run executes eagerly and sizes
 * every lane's scratch, and every later run replays the whole batch as ONE
 * CUDA-graph launch on `stream`.  No FP64 Ψ is written.  With a split
 * precision each snapshot runs the sparse mode products of
 * fcb200_snapshot_lj; the sparse tables' capacity is fixed
 * on the host when the snapshot is added (its largest neighbourhood within
 * r_cut + 0.1 Å, plus 4 atoms) and re-checked by fcb200_batch_set_positions,
 * which re-plans the batch when positions outgrow it.  k3_out must be device
 * memory ((3N)³ floats).
 */
typedef struct fcb200_batch* fcb200_batch_t;
int fcb200_batch_create(fcb200_handle h, int precision, size_t hbm_budget_bytes, fcb200_batch_t* out);
int fcb200_batch_add_lj(fcb200_batch_t b, const double* pos, int64_t n_atoms, const double* box,
                        double sigma, double eps, double r_cut, double tol, const double* masses,
                        const float* phi, float* k3_out);
int fcb200_batch_set_positions(fcb200_batch_t b, int64_t index, const double* pos, void* stream);
int fcb200_batch_run(fcb200_batch_t b, void* stream);
int fcb200_batch_info(fcb200_batch_t b, int64_t* n_snapshots, int64_t* lanes, int64_t* graph_nodes,
                      size_t* scratch_bytes);
/* The lane that runs snapshot `index` in the batch's current plan (made by the
 * first fcb200_batch_run after snapshots were added or re-planned;
 * FCB_ERR_ARG before that).  A lane runs its snapshots one after another, so
 * snapshots of one lane may share a K3 output buffer; snapshots of different
 * lanes run concurrently and must not. */
int fcb200_batch_lane(fcb200_batch_t b, int64_t index, int64_t* lane);
int fcb200_batch_destroy(fcb200_batch_t b);

/*
 * Device-side phase timing (no counterpart in the reference, which has no
 * instrumentation).  With profiling enabled, fcb200_snapshot_lj records CUDA
 * events on the caller's stream between its phases; fcb200_phase_times then
 * returns (waiting for the last event) up to 6 durations in ms:
 *   [0] pair tables + ASR self terms, [1] dense IFC3 write (+ fused mass-weighted
 *   operand), [2] φ split, [3] mode product 1, [4] mode product 2,
 *   [5] mode product 3.  A phase that did not run reports -1.
 */
int fcb200_set_profiling(fcb200_handle h, int enable);
int fcb200_phase_times(fcb200_handle h, double* ms, int max_phases);

/*
 * LJ IFC3 assembly that allocates no device memory (no counterpart in the
 * reference: it exists for callers that cannot let a library allocate).
 * A Julia host keeps device memory in CUDA.jl's pool, whose accounting never
 * sees allocations made inside a foreign library; programs that size all
 * device memory at start-up have the same rule; and cudaFree synchronises the
 * whole device, stalling callers that keep several streams busy.
 *
 * Same results as fcb200_third_order_lj (bit for bit), with these differences:
 *  - no handle; pos, masses, psi_out and psi32_mw_out must be device memory,
 *    box is a host array of 3 doubles;
 *  - n_atoms <= FCB_NOALLOC_MAX_ATOMS, otherwise FCB_ERR_ARG before any work;
 *  - its scratch is one fixed device array (about 14.3 MB) that every GPU
 *    loading the library keeps until the process exits.  All calls share it
 *    and it keeps the last call's contents (nothing in it needs to start at
 *    zero); calls that overlap on the GPU race on it and must be serialised;
 *  - the first call on a device looks up the array's address with that device
 *    current (again after the device's context was reset: the address is
 *    cached per CUDA context); make that first call before any stream capture
 *    begins.
 * Asynchronous on `stream`.
 */
#define FCB_NOALLOC_MAX_ATOMS 256
int fcb200_third_order_lj_noalloc(const double* pos, int64_t n_atoms, const double* box,
                                  double sigma, double eps, double r_cut, double tol,
                                  const double* masses, double* psi_out, float* psi32_mw_out,
                                  int flags, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FCB200_H */
