/*
 * hf_b200 — C ABI of the B200 (sm_100a) Fock-build / HF-objective library.
 *
 * Conventions
 *  - Every entry point returns an int status (HF_OK == 0).  On failure
 *    hf_last_error() returns a message for the calling thread.
 *  - All array pointers are DEVICE pointers owned by the caller, in the
 *    reference's row-major layouts:  P, h, refP, Sigma, F, Q: (nk1, nk2, nb, nb)
 *    complex; p, eps: (nk1, nk2, nb) real; w2d: (nk1, nk2) real; VR:
 *    (nk1, nk2, 1, 1) or (nk1, nk2, nb, nb), complex or real.  Complex values
 *    are interleaved (re, im).  "dtype" selects the storage precision:
 *    HF_C128 (complex128 / float64) or HF_C64 (complex64 / float32).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  No entry point
 *    synchronises the stream; results are ready when the stream reaches them.
 *  - Scratch memory is caller-provided ("workspace"); query its size first.
 *    No entry point allocates device memory.
 */
#ifndef HF_B200_H
#define HF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define HF_OK 0
#define HF_ERR_INVALID 1     /* bad argument or shape (the reference raises ValueError) */
#define HF_ERR_UNSUPPORTED 2 /* size outside what this build implements           */
#define HF_ERR_CUDA 3        /* a CUDA call or kernel launch failed               */
#define HF_ERR_WORKSPACE 4   /* workspace missing or too small                    */
#define HF_ERR_NONFINITE 5   /* non-finite value detected                         */
#define HF_ERR_MAXITER 6     /* iteration cap reached (solver did not converge)   */
#define HF_ERR_ABORTED 7     /* host abort flag was set                           */

/* ---- storage precision ---------------------------------------------------- */
#define HF_C128 0
#define HF_C64 1

/* ---- Fock-build flags ----------------------------------------------------- */
#define HF_FOCK_EXCHANGE (1u << 0)  /* include_exchange                                */
#define HF_FOCK_HARTREE (1u << 1)   /* include_hartree                                 */
#define HF_FOCK_PACKING (1u << 2)   /* exchange_hermitian_channel_packing (scalar VR)  */
#define HF_FOCK_VR_SCALAR (1u << 3) /* VR has shape (nk1, nk2, 1, 1)                   */
#define HF_FOCK_VR_REAL (1u << 4)   /* VR is stored as a real array                    */
#define HF_FOCK_FFT_FP32 (1u << 5)  /* complex128 storage, exchange FFT in FP32        */
#define HF_FOCK_HAS_REFP (1u << 6)  /* refP is non-zero and must be subtracted         */
#define HF_FOCK_GENERIC_FFT (1u << 7) /* force the generic shared-memory FFT engine    */
/* V_ab(q) is real and V_ab = V_ba (caller asserts): with HF_FOCK_PACKING the
 * Hermitian channel packing then also applies to a band-resolved V (only the
 * upper-triangle channels are transformed, Sigma_ba = conj(Sigma_ab)); exact
 * for a Hermitian density.  The reference packs scalar V only (utils.py:140-161). */
#define HF_FOCK_SYM_V (1u << 8)
/* Use the transpose-closed 2x2-tile slot groups in the fast engine even where
 * the rows plan would apply (nb <= 8 without packing); a schedule choice, the
 * result is the same to rounding. */
#define HF_FOCK_TILE_PLAN (1u << 9)
/* Run the rows plan (nb in {4, 8}, register mesh lengths, 16-byte aligned
 * operands) on the bulk-copy pipeline: one persistent CTA per SM, a ring of
 * shared-memory stages filled by tensor / bulk copies, Sigma and the
 * hermitised F in separate passes.  A schedule choice (the result is the same
 * to rounding); the autotuner times it as a candidate. */
#define HF_FOCK_PIPE (1u << 10)
const char* hf_last_error(void);
const char* hf_status_string(int status);
int hf_version(void);

/* ---- Fock build ------------------------------------------------------------
 * Replaces jax_hf.fock.build_fock (fock.py:18-97) -> utils.selfenergy_fft
 * (utils.py:66-173) for block_specs=None and project_fn=None.
 *   Sigma = -IFFT2(FFT2(P - refP) * VR) [+ contact sigma]     (all nb^2 channels, or
 *           the upper triangle + conjugate when HF_FOCK_PACKING)
 *   H     = diag(HH @ n), n_a = sum_k w_k Re(P - refP)_aa      (written as nb x nb; may be NULL)
 *   F     = herm(h + Sigma + H)
 * Contact terms (fock.py:77-92) are applied when n_contact > 0.
 * HH, w2d, contact_g are real at the storage precision; contact_Oi/Oj complex (t, nb, nb).
 * The exchange FFT runs on device in three passes (row FFT, column FFT x VR x
 * column IFFT, row IFFT + fused epilogue) through `workspace`.
 */
int hf_fock_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb, size_t* bytes);

int hf_fock_build(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                  const void* P, const void* h, const void* VR, const void* refP,
                  const void* HH, const void* w2d, int n_contact, const void* contact_g,
                  const void* contact_Oi, const void* contact_Oj, void* Sigma, void* H, void* F,
                  void* workspace, size_t workspace_bytes);

/* Same Fock build as hf_fock_build, for callers that cannot allocate device
 * memory (a framework custom-call handler that owns all device buffers, code
 * running under CUDA stream capture): the scratch is a library-owned static
 * device array of HF_FOCK_STATIC_SCRATCH_BYTES, so no workspace argument.
 * No counterpart in the reference (jax_hf allocates through XLA).
 *  - Returns HF_ERR_WORKSPACE if the mesh needs more scratch than the array
 *    holds (hf_fock_workspace_size() > HF_FOCK_STATIC_SCRATCH_BYTES; e.g. up
 *    to 192x192 with nb = 8 in complex128).
 *  - The first call in a CUDA context looks up the array's device address
 *    (cached under the context's unique id); make it before any stream
 *    capture.  The array stays allocated while the context lives; after a
 *    cudaDeviceReset the next call looks the address up again.
 *  - All calls on a device share the array: calls that may overlap on the GPU
 *    race and must be serialised by the caller. */
#define HF_FOCK_STATIC_SCRATCH_BYTES (40u << 20)
int hf_fock_build_static_scratch(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                                 const void* P, const void* h, const void* VR, const void* refP,
                                 const void* HH, const void* w2d, int n_contact, const void* contact_g,
                                 const void* contact_Oi, const void* contact_Oj, void* Sigma, void* H,
                                 void* F);

/* Block-diagonal exchange (utils.py:206-309, build_fock with exchange_block_specs):
 * the same outputs as hf_fock_build except that the exchange self-energy is
 * formed only on the in-block channels of `inblock` (HOST, nb x nb bytes,
 * symmetric, nonzero = in-block: the channels (a, b) with a and b in one block)
 * and is zero on the others.  Only in-block channels are transformed, so the
 * exchange passes do (in-block channels / nb^2) of the full work; the Hartree and
 * contact terms still see every channel of P - refP, as in fock.py:66-92.
 * Workspace: hf_fock_blocks_workspace_size (depends on the mask).  Without
 * HF_FOCK_EXCHANGE or with every channel in-block this is hf_fock_build.
 *
 * hf_block_offdiag_max: out (DEVICE, n_specs + 1 float64) = { max |P - refP|,
 * then for each spec i the max of |P - refP| over its off-block channels }, with
 * inblock holding n_specs masks back to back (HOST; n_specs <= 8, nb <= 32;
 * refP may be NULL).  One pass over P, no host synchronisation: the caller
 * reads the n_specs + 1 values once and takes the first spec whose off-block
 * maximum is <= atol + rtol * max (utils.py:263-267); NaN propagates. */
int hf_fock_blocks_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb,
                                  const unsigned char* inblock, size_t* bytes);
int hf_fock_build_blocks(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                         const unsigned char* inblock, const void* P, const void* h, const void* VR,
                         const void* refP, const void* HH, const void* w2d, int n_contact, const void* contact_g,
                         const void* contact_Oi, const void* contact_Oj, void* Sigma, void* H, void* F,
                         void* workspace, size_t workspace_bytes);
int hf_block_offdiag_max(void* stream, int dtype, size_t nk, int nb, const void* P, const void* refP, int n_specs,
                         const unsigned char* inblock, double* out);

/* build_fock with exchange_block_specs and check_offdiag (utils.py:252-309) without a
 * host round trip: hf_block_offdiag_max, then a one-thread kernel picks the first
 * compatible spec (or the full build) and sets a device flag; the masked build of
 * every spec and the full build are all queued, and the kernels of every candidate
 * but the chosen one return at once.  inblock: n_specs (1..8) masks back to back
 * (HOST).  chosen (DEVICE int, may be NULL) receives the spec index or -1 for the
 * full build.  Workspace: hf_fock_block_specs_workspace_size. */
int hf_fock_block_specs_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb, int n_specs,
                                       const unsigned char* inblock, size_t* bytes);
int hf_fock_build_block_specs(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, int n_specs,
                              const unsigned char* inblock, double atol, double rtol, const void* P, const void* h,
                              const void* VR, const void* refP, const void* HH, const void* w2d, int n_contact,
                              const void* contact_g, const void* contact_Oi, const void* contact_Oj, void* Sigma,
                              void* H, void* F, void* workspace, size_t workspace_bytes, int* chosen);

/* Autotuner for the Fock-build schedule (slot plan and FFT engine per shape;
 * no counterpart in the reference, whose FFTs are XLA's).  Same arguments as
 * hf_fock_build, plus reps (timed builds
 * per candidate, >= 1), chosen (out: the engine flags picked) and us (out,
 * may be NULL, 4 entries: mean microseconds per build of each candidate, in
 * the order default schedule / HF_FOCK_TILE_PLAN / HF_FOCK_GENERIC_FFT /
 * HF_FOCK_PIPE, -1 for a candidate that does not apply).  Every candidate runs on the caller's
 * buffers (one untimed build, then reps timed with CUDA events on `stream`),
 * the fastest is stored in a process-wide table keyed by (device, dtype,
 * flags, nk1, nk2, nb), and the outputs hold the winner's result on return.
 * Later hf_fock_build calls with the same key and no engine flag of their own
 * (HF_FOCK_TILE_PLAN, HF_FOCK_GENERIC_FFT), including those made inside the
 * solver drivers, use the stored choice.  Synchronises `stream`: call it
 * outside stream capture.  The workspace must hold
 * hf_fock_workspace_size(), which covers every candidate. */
int hf_fock_autotune(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                     const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                     int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                     void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes, int reps,
                     unsigned* chosen, float* us);
/* Forgets every stored autotuner choice. */
int hf_fock_autotune_reset(void);

/* Device fault word of the pipelined Fock passes on the current device (no
 * counterpart in the reference).  Every wait of those kernels on an mbarrier
 * is bounded (2 s); one that runs out records a nonzero code (2: a consumer
 * group waiting for a stage's copy, 3: waiting for the copy to be issued) and
 * the kernel returns without finishing the build.  Synchronises the device, copies
 * the word to *code and, when clear != 0, resets it to zero. */
int hf_fock_fault_status(int* code, int clear);

/* Periodic linear resampling of the two leading axes of an (n1, n2, ...)
 * array on a centered k-grid (k = 0 at index n / 2) to (m1, m2, ...):
 * utils.py:477-535 (resample_kgrid, method "linear"), axis 0 then axis 1,
 * positions and weights in the array's real precision.  dtype HF_C128 for
 * float64 / complex128 data, HF_C64 for float32 / complex64; ncomp = real
 * components per k-point (2 x elements for complex data).  x and y must not
 * alias. */
int hf_resample_kgrid(void* stream, int dtype, int n1, int n2, int m1, int m2, long long ncomp, const void* x,
                      void* y);
/* The continuation driver's density seed (continuation.py:47-50):
 * out = (Q + Q^H) / 2 with Q = resample_kgrid(P), P (n1, n2, nb, nb) complex. */
int hf_resample_density(void* stream, int dtype, int n1, int n2, int m1, int m2, int nb, const void* P, void* out);

/* Symmetry averaging of (nk1, nk2, nb, nb) matrices (symmetry.py:22-150, the
 * building blocks of make_project_fn; nb <= 32, dtype HF_C128 or HF_C64).
 * k-point maps: HF_K_FLIP (i -> n - 1 - i, jnp.flip), HF_K_MOD (i -> -i mod n)
 * on the axes whose bit is set in flip_axes (bit 0: axis 0, bit 1: axis 1), or
 * HF_K_INDEX_MAP (k -> (idx_i[k], idx_j[k]) from per-element int32 tables).
 * Index-map entries must lie in [0, nk1) x [0, nk2); an entry outside is
 * read as the identity map (no out-of-bounds access).  A and out must not
 * alias. */
#define HF_K_FLIP 0
#define HF_K_MOD 1
#define HF_K_INDEX_MAP 2
/* out(k) = (sum_{g<n_same} G_same[g] A(k) G_same[g]^H
 *          + sum_{g<n_mapped} G_mapped[g] A(map_g(k)) G_mapped[g]^H) / (n_same + n_mapped);
 * index maps idx_i, idx_j: (n_mapped, nk1, nk2).  mask (nk1, nk2) bytes or NULL:
 * where 0, out(k) = A(k) (spatial_k_orbit_mask). */
int hf_sym_group_average(void* stream, int dtype, int nk1, int nk2, int nb, const void* A, void* out, int n_same,
                         const void* G_same, int n_mapped, const void* G_mapped, int k_mode, int flip_axes,
                         const int* idx_i, const int* idx_j, const unsigned char* mask);
/* out(k) = (A(k) + U conj(A(-k)) U^H) / 2 with -k from the k-map (index map
 * (nk1, nk2) tables); with HF_K_INDEX_MAP, out(k) = A(k) where valid[k] == 0. */
int hf_sym_time_reversal(void* stream, int dtype, int nk1, int nk2, int nb, const void* A, void* out, const void* U,
                         int k_mode, int flip_axes, const int* idx_i, const int* idx_j, const unsigned char* valid);

/* Superlattice Fock exchange on the extended momentum grid (superlattice.py:
 * 167-229, make_superlattice_fock_fn), complex128: rho and sigma are
 * (nkx, nky, n_G dim_orb, n_G dim_orb); V_lag_fft is (N_ext_x, N_ext_y)
 * complex128 (the layout's FFT of the lag Coulomb kernel); g_a_off (n_G, 2)
 * int32 tile offsets; pair_to_delta (n_G, n_G) int32 DG index of each pair;
 * tile_owner (n_delta, N_ext_x / nkx, N_ext_y / nky) int32: i n_G + j of the
 * pair (i, j) of that DG whose tile sits there, or -1.  All DG channels are
 * transformed with the library's exchange build in chunks of up to 1024
 * channels; workspace from hf_sl_fock_workspace_size. */
int hf_sl_fock_workspace_size(int nkx, int nky, int n_G, int dim_orb, int N_ext_x, int N_ext_y, int n_delta,
                              size_t* bytes);
int hf_sl_fock(void* stream, int nkx, int nky, int n_G, int dim_orb, int N_ext_x, int N_ext_y, int n_delta,
               const int* tile_owner, const int* g_a_off, const int* pair_to_delta, const void* V_lag_fft,
               const void* rho, void* sigma, void* workspace, size_t workspace_bytes);

/* ---- Objective reductions (compensated, FP64 accumulation) -----------------
 * hf_energy replaces fock.hf_energy (fock.py:100-111):
 *   E = sum_k w_k Re Tr[(h + (Sigma + H)/2) P]
 * H_mode: 0 = no H, 1 = H is one nb x nb matrix for all k, 2 = H per k.
 * hf_occupation_entropy replaces fock.occupation_entropy (fock.py:114-118);
 * hf_free_energy replaces fock.free_energy (fock.py:121-129) with E read from
 * device memory.  Scalar outputs are float64 device pointers.
 */
int hf_reduce_workspace_size(int nk1, int nk2, int nb, size_t* bytes);
int hf_energy(void* stream, int dtype, int nk1, int nk2, int nb, const void* P, const void* h,
              const void* Sigma, const void* H, int H_mode, const void* w2d, double* E_out,
              void* workspace, size_t workspace_bytes);
int hf_occupation_entropy(void* stream, int dtype, int nk1, int nk2, int nb, const void* p,
                          const void* w_norm, double* S_out, void* workspace,
                          size_t workspace_bytes);
int hf_free_energy(void* stream, int dtype, int nk1, int nk2, int nb, const double* E,
                   const void* p, const void* w_norm, double T, double* Omega_out,
                   void* workspace, size_t workspace_bytes);

/* ---- Chemical potential ------------------------------------------------------
 * method 0: pure bisection            utils._find_mu_bisection (utils.py:353-382)
 * method 1: Newton with bracket       utils._find_mu_newton    (utils.py:385-442)
 * method 2: Newton-bracket from mu0   solver._solve_mu         (solver.py:62-101)
 * maxiter <= 0 picks the reference default for the method and dtype.
 * weights: method 0/1 take raw weights and n_electrons; method 2 takes the
 * normalised weights and n_target_norm (as the solver does).  mu0 (device,
 * float64, may be NULL) is method 2's warm start and, for method 0, a hint (a
 * previous mu): Newton passes from it certify a bracket around the root, and
 * the bisection levels whose midpoints lie outside it are decided without
 * evaluations, with the decisions, and so the result, of evaluating every
 * level; method 1 ignores it.  mu0 may alias mu_out.  mu_out is a float64
 * device scalar.
 */
int hf_find_mu(void* stream, int dtype, int method, int nk1, int nk2, int nb, const void* eps,
               const void* weights, double n_electrons, double T, int maxiter, const double* mu0,
               double* mu_out);

/* ---- Per-k small matrices (one warp per k-point) ------------------------------
 * batch = number of nb x nb matrices (nk1*nk2 for mesh arrays).
 * hf_density_from_Qp:   P = herm(Q diag(p) Q^H)            solver.py:42-44 (+ _herm)
 * hf_fock_orbital:      Ft = Q^H F Q                        solver.py:47-49
 * hf_eigh:              A = V diag(w) V^H, w ascending       jnp.linalg.eigh (LAPACK heevd)
 * hf_cayley_retract:    U = (I + tau d/2)^-1 (I - tau d/2)   solver.py:122-138 (tau on host)
 * hf_cayley_spectral:   (V, lam) = eigh(herm(i d))           solver.py:161-166
 * hf_cayley_unitary:    U = V diag(c(tau, lam)) V^H          solver.py:169-182
 * hf_diag_UFU:          diag(U^H Ft U) from V, Ft_eig, lam   solver.py:185-197
 * hf_qr_retract:        U = QR(I - tau G), phase-fixed       solver.py:108-119
 * Real outputs (w, lam, p, diag) are at the storage precision.
 */
int hf_density_from_Qp(void* stream, int dtype, int batch, int nb, const void* Q, const void* p,
                       void* P);
int hf_fock_orbital(void* stream, int dtype, int batch, int nb, const void* Q, const void* F,
                    void* Ft);
int hf_eigh(void* stream, int dtype, int batch, int nb, const void* A, void* w, void* V);
/* Extension (no counterpart in the reference): complex128 eigendecomposition of nk
 * Hermitian nb x nb matrices (nb <= 8; A hermitised) by a lane-per-column cyclic
 * Jacobi, eigenvalues ascending in w, eigenvectors as the columns of Qout.  With a
 * starting basis Qin (may be NULL; may equal Qout) the rotation is applied to
 * Qin^H A Qin and Qout = Qin V: when Qin already diagonalises a nearby matrix (the
 * previous SCF iteration's Fock matrix), the sweeps converge at once.  The result
 * is an exact decomposition either way (to the Jacobi tolerance). */
int hf_eigh_warm(void* stream, int nk, int nb, const void* A, const void* Qin, void* Qout, void* w);
int hf_cayley_retract(void* stream, int dtype, int batch, int nb, const void* d, double tau,
                      void* U);
int hf_cayley_spectral(void* stream, int dtype, int batch, int nb, const void* d, void* V,
                       void* lam);
int hf_cayley_unitary(void* stream, int dtype, int batch, int nb, const void* V, const void* lam,
                      double tau, void* U);
int hf_diag_UFU(void* stream, int dtype, int batch, int nb, const void* V, const void* Ft_eig,
                const void* lam, double tau, void* diag);
int hf_qr_retract(void* stream, int dtype, int batch, int nb, const void* G, double tau,
                  void* U);

/* ---- Solver building blocks (complex128 / float64) ----------------------------
 * Used by the SCF loop (reference_scf.py:222-365) and the trust-region Newton
 * loop (solver.py:686-1078).  Reductions write float64 results to device
 * memory; `ws` is scratch of hf_ops_workspace_size() bytes.
 *  hf_fermi          mode 0: fermidirac(eps-mu, T) (utils.py:51-53); mode 1: sigmoid((mu-eps)/max(T,1e-12))
 *                    (solver.py:394); mode 2: eps + shift (1 - fermidirac(eps-mu, T)) (reference_scf.py:92).
 *                    mu is a device scalar.
 *  hf_scf_residuals  comm = F P - P F, delta = Pn - P and sums3 = {sum w|delta|^2, sum w|comm|^2,
 *                    sum w Re tr(F delta)}  (reference_scf.py:291-295, 319-320)
 *  hf_gram           DIIS B_ij = sum_k w Re tr(R_i^H R_j), upper triangle row-major (reference_scf.py:110-111)
 *  hf_gram_row       b_j = B_ij for one i and every j < n (n <= 16): the row of B that changes when DIIS
 *                    replaces history slot i; each entry equals hf_gram's bit for bit (extension, no
 *                    reference counterpart; the reference recomputes all of B each step)
 *  hf_lincomb        out = sum_i c_i X_i, c on device (reference_scf.py:305)
 *  hf_axpby          out = [herm](a x + b y); hf_axpby_real the same for real vectors
 *  hf_jdot           sum_k wX sum Re(conj(aX) bX) + sum_k wp sum ap bp (solver.py:205-233, 783-787)
 *  hf_orbital_grad   G = skew((p_j - p_i) Ft) offdiag, eps = Re diag Ft (solver.py:898-900)
 *  hf_newton_prec    z = (rX / sqrt(gap^2 + lam^2), rp p(1-p)/T) + sum w2d zp (solver.py:907-913)
 *  hf_sub_scalar     x -= scale * c[0]   (particle-number projection, solver.py:224-233)
 *  hf_newton_dP      dP = herm(Q (X o dpij + diag dp) Q^H) (solver.py:917-919)
 *  hf_newton_hvp     HX, Hp of the joint Hessian from Fr = F[dP] (solver.py:920-930)
 *  hf_matmul, hf_real_diag  per-k C = A B, d = Re diag A
 */
int hf_ops_workspace_size(size_t* bytes);
int hf_fermi(void* stream, size_t n, const double* eps, const double* mu, double T, int mode, double shift,
             double* out);
int hf_scf_residuals(void* stream, int nk, int nb, const void* F, const void* P, const void* Pn, const double* w,
                     void* comm, void* delta, double* sums3, void* ws);
int hf_gram(void* stream, int n, size_t stride, int nk, int nb, const void* R, const double* w, double* B_out,
            void* ws);
int hf_gram_row(void* stream, int n, int i, size_t stride, int nk, int nb, const void* R, const double* w,
                double* b_out, void* ws);
int hf_lincomb(void* stream, int n, size_t stride, size_t len, const void* X, const double* c, void* out);
int hf_axpby(void* stream, size_t nk, int nb, double a, const void* x, double b, const void* y, int herm,
             void* out);
int hf_axpby_real(void* stream, size_t n, double a, const double* x, double b, const double* y, double* out);
int hf_jdot(void* stream, size_t nk, int nb, const void* aX, const void* bX, const double* wX, const double* ap,
            const double* bp, const double* wp, double* out, void* ws);
int hf_orbital_grad(void* stream, size_t nk, int nb, const void* Ft, const double* p, void* G, double* eps);
int hf_newton_prec(void* stream, size_t nk, int nb, const void* rX, const double* rp, const double* eps,
                   const double* p, double lam, double T, double clipv, const double* w2d, void* zX, double* zp,
                   double* wsum_out, void* ws);
int hf_sub_scalar(void* stream, size_t n, double* x, const double* c, double scale);
int hf_newton_dP(void* stream, int nk, int nb, const void* Q, const void* X, const double* dp, const double* p,
                 void* dP);
int hf_newton_hvp(void* stream, int nk, int nb, const void* Q, const void* Ft, const void* X, const double* dp,
                  const double* p, const void* Fr, const void* h, double T, double clipv, double pen,
                  const void* dPpen, void* HX, double* Hp, const double* w2d, double* wsum_out, void* ws);
int hf_matmul(void* stream, int nk, int nb, const void* A, const void* B, void* C);
int hf_real_diag(void* stream, size_t nk, int nb, const void* A, double* d);

/* ---- Device-resident solvers ---------------------------------------------------
 * The problem is a HartreeFockKernel's arrays (problem.py:201-217 as_args) in
 * complex128 storage.  fock_flags carries HF_FOCK_EXCHANGE/HARTREE/PACKING/
 * VR_SCALAR/VR_REAL/HAS_REFP exactly as for hf_fock_build.
 */
/* Optional host callbacks of the CG driver, invoked when an iteration is
 * enqueued (they must enqueue their device work on `stream` and return an
 * hf status): fock_cb replaces the built-in Fock build (Sigma, H (nb x nb), F
 * from P), project_cb maps P -> herm(project(P)) in place. */
typedef int (*hf_fock_callback)(void* user, void* stream, const void* P, void* Sigma, void* H, void* F);
typedef int (*hf_project_callback)(void* user, void* stream, void* P);

typedef struct hf_cg_problem {
  int nk1, nk2, nb;
  unsigned fock_flags;
  double T, n_electrons, weight_sum;
  const void* h;          /* (nk1, nk2, nb, nb) complex128                 */
  const void* VR;         /* phase-shifted VR (complex128 or float64)       */
  const void* refP;       /* may be NULL unless HF_FOCK_HAS_REFP            */
  const void* HH;         /* (nb, nb) float64, may be NULL without Hartree  */
  const void* w2d;        /* (nk1, nk2) float64 raw weights                 */
  int n_contact;
  const void* contact_g;  /* (t,) float64                                   */
  const void* contact_Oi; /* (t, nb, nb) complex128                         */
  const void* contact_Oj;
  void* sigma_buf;        /* optional caller buffer for Sigma (nk1, nk2, nb, nb) */
  void* h_buf;            /* optional caller buffer for H (nb, nb)               */
} hf_cg_problem;

/* SolverConfig fields (solver.py:240-286) plus the mixed-precision policy:
 * fp32_exchange != 0 runs the exchange FFT in FP32 until the windowed energy
 * change reaches fp32_switch_rel*|E| (or half of max_iter), then continues with
 * FP64 builds (defect correction) to tol_E / tol_grad; the final builds are FP64.
 * chunk = iterations queued between host checks of the device stop flag. */
typedef struct hf_cg_config {
  int max_iter;
  double tol_E, tol_grad, denom_scale, max_step;
  int cg_restart;
  double bt_shrink;
  int bt_max, mu_maxiter, plateau_window;
  int fp32_exchange;
  double fp32_switch_rel;
  int chunk;
  hf_fock_callback fock_cb;       /* NULL: built-in hf_fock_build */
  hf_project_callback project_cb; /* NULL: no projection           */
  void* cb_user;
} hf_cg_config;

/* Direct-minimisation CG (solver.py:307-660, optimizer="cg"): replaces
 * jax_hf.solve / solve_direct_minimization for project_fn=None, block_sizes=None.
 * Inputs: P0 (nk1, nk2, nb, nb) complex128.  Outputs (device): Q, p, density,
 * fock as in SolveResult; hist_E / hist_grad (max_iter float64, may be NULL);
 * scalars_out (8 float64): mu, energy, n_iter, converged, last grad_norm,
 * iteration of the FP32->FP64 switch (-1 if none), 0, 0.
 * Synchronises `stream` once per chunk of iterations and at the end. */
int hf_cg_workspace_size(const hf_cg_problem* problem, const hf_cg_config* config, size_t* bytes);
int hf_cg_solve(void* stream, const hf_cg_problem* problem, const hf_cg_config* config, const void* P0,
                void* Q, void* p, void* density, void* fock, double* hist_E, double* hist_grad,
                double* scalars_out, void* workspace, size_t workspace_bytes);

/* ---- SCF driver (complex128) ---------------------------------------------------
 * Replaces jax_hf.reference_scf.solve_scf (reference_scf.py:124-365) for
 * project_fn=None and the built-in Fock build: Roothaan iteration with linear
 * mixing (acceleration 0), Pulay C-DIIS (1) or ODA (2), level shift and
 * trust-radius clip; SCFConfig fields and defaults as reference_scf.py:31-63
 * (diis_size <= 16).  The problem is described by an hf_cg_problem
 * (sigma_buf / h_buf unused).  Inputs: P0 (nk1, nk2, nb, nb) complex128.
 * Outputs: density and fock (device, as SCFResult.density_matrix /
 * fock_matrix), the per-iteration histories hist_E, hist_D, hist_C (HOST
 * float64, max_iter entries each, may be NULL) and scalars_out (HOST, 4
 * float64): energy, chemical potential, iterations, converged.  Synchronises
 * `stream` once per iteration (twice for ODA or a trust-radius clip).
 * Extensions (no counterpart in the reference; zero keeps its behaviour):
 *  - fp32_exchange != 0: mixed precision.  Builds run the exchange FFT in FP32
 *    (HF_FOCK_FFT_FP32) while the previous iteration's density residual exceeds
 *    fp32_switch_density; from the first iteration below it every build is FP64,
 *    the DIIS history restarts, and convergence is only declared on FP64 builds,
 *    so the result is the FP64 fixed point.  scalars_out then has a fifth entry:
 *    the first FP64 iteration (-1 if the FP32 phase never ended).
 *  - mu_method 2: the chemical potentials come from the Newton-bracket solver
 *    (solver.py:62-101 rules), started at mu = 0 in the first iteration and at
 *    the previous iteration's mu afterwards, instead of the 54-step bisection
 *    (the same root to rounding; level_shift must be 0).
 *  - warm_eigh != 0 (nb <= 8): the eigendecompositions of the iterations after
 *    the first start from the previous iteration's eigenvectors (hf_eigh_warm);
 *    the same decomposition to the Jacobi tolerance, in fewer sweeps.
 * Hooks (solve_scf's fock_build_fn and project_fn, reference_scf.py:124-365): with
 * fock_cb the driver calls fock_cb(cb_user, stream, P, Sigma, H, F) for every build
 * instead of hf_fock_build (H: nb x nb; fp32_exchange is then refused); with
 * project_cb it calls project_cb(cb_user, stream, X) where the reference applies
 * herm(project(.)) instead of herm(.): X holds the unprojected array and the
 * callback replaces it in place by herm(project(X)) (the density before each build,
 * the built F, the new density, the DIIS density and the mixed density).  The
 * pointers are the driver's buffers inside the caller's workspace or outputs; a
 * callback enqueues its work on `stream` and returns 0, or nonzero to abort
 * (HF_ERR_ABORTED). */
typedef struct hf_scf_config {
  int max_iter;
  double density_tol, comm_tol, mixing, level_shift;
  int acceleration; /* 0 linear, 1 diis, 2 oda */
  int diis_size, diis_start;
  double diis_damping, trust_radius;
  int fp32_exchange;          /* extension, see above */
  double fp32_switch_density; /* extension */
  int mu_method;              /* extension: 0 bisection (reference), 2 Newton-bracket warm start */
  int warm_eigh;              /* extension: eigh from the previous iteration's eigenvectors (nb <= 8) */
  hf_fock_callback fock_cb;       /* NULL: built-in hf_fock_build */
  hf_project_callback project_cb; /* NULL: no projection           */
  void* cb_user;
} hf_scf_config;

int hf_scf_workspace_size(const hf_cg_problem* problem, const hf_scf_config* config, size_t* bytes);
int hf_scf_solve(void* stream, const hf_cg_problem* problem, const hf_scf_config* config, const void* P0,
                 void* density, void* fock, double* hist_E, double* hist_D, double* hist_C, double* scalars_out,
                 void* workspace, size_t workspace_bytes);

/* A batch of independent SCF solves as ONE CUDA graph (extension, no reference
 * counterpart): the loop of hf_scf_solve with its decisions on the device, so that no
 * host round trip happens between the launch and the end of the last solve.  Every
 * solve is a branch: init -> iteration 0 -> [WHILE FP32 iterations -> switch] ->
 * WHILE FP64 iterations -> final FP64 build; the DIIS bordered system is solved by a
 * one-thread kernel with the host driver's LU, and DIIS-or-mixing is a conditional IF
 * node.  DIIS and linear mixing with every hf_scf_config option except ODA
 * (acceleration 2) and the trust-radius clip (HF_ERR_UNSUPPORTED: they read values
 * on the host every iteration).  Items: the problem, P0, the outputs (density, fock),
 * per-iteration histories (DEVICE, max_iter float64 each, may be NULL) and scalars_out
 * (DEVICE, 5 float64: energy, mu, iterations, converged, first FP64 iteration or -1).
 * The workspace holds n_items blocks of bytes_per_item (hf_scf_batch_workspace_size).
 * _create captures and instantiates (host work only), _launch runs the graph after
 * the work queued on `stream` (solve_ms, may be NULL: waits and fills each solve's
 * time), _destroy frees it; new starting densities may be written to the P0 buffers
 * between launches. */
typedef struct hf_scf_batch_item {
  hf_cg_problem problem;
  const void* P0;
  void* density;
  void* fock;
  double* hist_E;
  double* hist_D;
  double* hist_C;
  double* scalars_out;
} hf_scf_batch_item;

int hf_scf_batch_workspace_size(const hf_scf_batch_item* items, int n_items, const hf_scf_config* config,
                                size_t* bytes_per_item);
int hf_scf_batch_graph_create(const hf_scf_batch_item* items, int n_items, const hf_scf_config* config,
                              void* workspace, size_t bytes_per_item, void** handle);
int hf_scf_batch_graph_launch(void* handle, void* stream, double* solve_ms);
int hf_scf_batch_graph_destroy(void* handle);

/* ---- Trust-region Newton driver (complex128) -----------------------------------
 * Replaces jax_hf.solve with optimizer="newton" (solver.py:686-1078) for
 * project_fn=None, block_sizes=None and the built-in Fock build (nb <= 16):
 * Steihaug truncated CG on the joint (Q, p) Hessian, Cayley trial steps,
 * trust-region updates and the Gaussian deflation bias (solver.py:799-812).
 * SolverConfig fields as solver.py:240-286; tol_grad <= 0 means 1e-6
 * (solver.py:1191).  deflation_targets: n_deflation (nk1, nk2, nb, nb)
 * complex128 device arrays back to back (used when n_deflation > 0 and
 * deflation_sigma > 0).  The problem is an hf_cg_problem (sigma_buf / h_buf
 * unused).  Outputs: Q (nk1, nk2, nb, nb) complex128, p (nk1, nk2, nb) float64,
 * density and fock (device, as SolveResult), hist_E / hist_G (HOST float64,
 * max_iter entries, may be NULL) and scalars_out (HOST, 6 float64): mu,
 * energy, n_iter, converged, last grad_norm, Fock builds.  The host reads the
 * loop's reductions in small batches: two reads per inner CG step, three or
 * four per outer step. */
typedef struct hf_newton_config {
  int max_iter;
  double tol_grad, denom_scale;
  int mu_maxiter;
  double tr_delta0;
  int tr_cg_max;
  int n_deflation;
  const void* deflation_targets;
  double deflation_sigma, deflation_length;
} hf_newton_config;

int hf_newton_workspace_size(const hf_cg_problem* problem, const hf_newton_config* config, size_t* bytes);
int hf_newton_solve(void* stream, const hf_cg_problem* problem, const hf_newton_config* config, const void* P0,
                    void* Q, void* p, void* density, void* fock, double* hist_E, double* hist_G,
                    double* scalars_out, void* workspace, size_t workspace_bytes);

/* ---- Reverse mode (complex128) -------------------------------------------------
 * The reference differentiates build_fock / hf_energy / free_energy with
 * jax.grad (fock.py:18-129 under jax autodiff); these are the hand-written
 * adjoints behind the PyTorch autograd Functions of adjoint.py.  Gradients
 * use torch's convention for complex leaves (d/dRe + i d/dIm).
 *
 * hf_fock_build_vjp: cotangents Sigma_bar, F_bar (either may be NULL) of the
 * (Sigma, F) outputs of hf_fock_build -> P_bar = A^H(Sigma_bar + herm(F_bar))
 * with A^H the exchange map run with VR_adj = conj(VR) (VR itself when real),
 * and h_bar = herm(F_bar) (may be NULL).  Exchange part only: the Hartree and
 * contact terms are linear maps of a few nb x nb reductions and are
 * differentiated by the caller.  Workspace from hf_fock_vjp_workspace_size. */
int hf_fock_vjp_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb, size_t* bytes);
int hf_fock_build_vjp(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* Sigma_bar,
                      const void* F_bar, const void* VR_adj, void* P_bar, void* h_bar, void* workspace,
                      size_t workspace_bytes);
/* hf_energy_vjp: E = Re sum_k w_k tr((h + (Sigma + H)/2) P) with cotangent E_bar ->
 * P_bar = E_bar w (h + (Sigma+H)/2)^H, h_bar = E_bar w P^H, Sigma_bar = E_bar w P^H / 2
 * (each output may be NULL).  H_mode as hf_energy. */
int hf_energy_vjp(void* stream, int nk1, int nk2, int nb, const void* P, const void* h, const void* Sigma,
                  const void* H, int H_mode, const double* w2d, double E_bar, void* P_bar, void* h_bar,
                  void* Sigma_bar);
/* hf_free_energy_vjp: Omega = E - max(T,1e-14) S(p) -> p_bar = Omega_bar T w_norm (log p - log1p(-p))
 * inside the entropy clip range [1e-14, 1-1e-14], 0 outside; E_bar = Omega_bar. */
int hf_free_energy_vjp(void* stream, int nk1, int nk2, int nb, const double* p, const double* w_norm, double T,
                       double Omega_bar, double* p_bar);
/* hf_fourier_coeffs: out[r] = sum_k w_k exp(-i k.R_r) P_k for nR lattice vectors R (int pairs), k on
 * the centred grid k_m = 2 pi (m - n/2) / n: the gradient of sum_k w_k Re tr(h_k P_k) with respect to
 * an independent Fourier coefficient h_R of h_k = sum_R h_R exp(i k.R) (P Hermitian).  No counterpart
 * in the reference (jax.grad through the user's Hamiltonian construction plays this role). */
int hf_fourier_coeffs(void* stream, int nk1, int nk2, int nb, const void* P, const double* w2d, int nR,
                      const int* R, void* out);

/* Batched density scan: many independent CG solves, no host callbacks.  The
 * solves are ordered longest first (nk * nb^2 * (nb + 8)) and run n_lanes at a
 * time, each lane on its own stream (ordered after `stream`, which waits for all
 * of them at the end) with its iterations replayed from CUDA graphs; the host
 * thread polls events and feeds a free lane the next solve.  Each item has the
 * outputs of hf_cg_solve.  workspace = n_lanes * bytes_per_lane bytes
 * (bytes_per_lane from hf_cg_batch_workspace_size).  solve_ms (host, n_items,
 * may be NULL) receives each solve's device time from its start to its final
 * scalars.  Extension of the reference API (the reference runs solves one by
 * one from Python, e.g. benchmarks/ and continuation.py loops). */
typedef struct hf_cg_batch_item {
  hf_cg_problem problem;
  const void* P0;
  void* Q;
  void* p;
  void* density;
  void* fock;
  double* hist_E;      /* may be NULL */
  double* hist_grad;   /* may be NULL */
  double* scalars_out; /* device, 8 float64 as for hf_cg_solve */
} hf_cg_batch_item;

int hf_cg_batch_workspace_size(const hf_cg_batch_item* items, int n_items, const hf_cg_config* config,
                               size_t* bytes_per_lane);
int hf_cg_solve_batch(void* stream, const hf_cg_batch_item* items, int n_items, const hf_cg_config* config,
                      int n_lanes, void* workspace, size_t bytes_per_lane, double* solve_ms);
/* The same batch as ONE CUDA graph, built and launched once: every solve is a branch
 * init -> iteration loop(s) -> finalize whose loops are conditional WHILE nodes, their
 * condition set on the device after every iteration, so nothing returns to the host
 * until the last solve ends.  All solves run at once: the workspace holds n_items
 * blocks of bytes_per_item (hf_cg_batch_workspace_size), one per solve.  Results equal
 * hf_cg_solve_batch's, except that the loop tests run after every iteration instead of
 * every `chunk` iterations (a mixed-precision solve that reaches half its iteration
 * budget in the FP32 phase switches at exactly max_iter / 2).  Extension. */
int hf_cg_solve_batch_graph(void* stream, const hf_cg_batch_item* items, int n_items, const hf_cg_config* config,
                            void* workspace, size_t bytes_per_item, double* solve_ms);
/* The same in three steps, for a scan run more than once: _create captures and
 * instantiates the graph (host work, no GPU work; the items' pointers are baked in),
 * _launch runs it after the work queued on `stream` and makes `stream` wait for it
 * (solve_ms, may be NULL: waits and fills each solve's time), _destroy frees it
 * (after waiting for a launch in flight).  Between launches the caller may write new
 * starting densities into the items' P0 buffers. */
int hf_cg_batch_graph_create(const hf_cg_batch_item* items, int n_items, const hf_cg_config* config, void* workspace,
                             size_t bytes_per_item, void** handle);
int hf_cg_batch_graph_launch(void* handle, void* stream, double* solve_ms);
int hf_cg_batch_graph_destroy(void* handle);

#ifdef __cplusplus
}
#endif

#endif /* HF_B200_H */
